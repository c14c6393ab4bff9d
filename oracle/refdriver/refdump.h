// Minimal tagged binary dump used by the oracle driver (test infrastructure).
//
// File layout: repeated records of
//   int32 name_len | name bytes | char kind ('d' float64, 'i' int32) | int64 count | payload
// Read by tests/refdump.py.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

class RefDump {
public:
	explicit RefDump(const std::string& path) { f_ = std::fopen(path.c_str(), "wb"); }
	~RefDump() { if (f_) std::fclose(f_); }
	bool ok() const { return f_ != nullptr; }
	void put(const std::string& name, const double* p, int64_t n) { head(name, 'd', n); std::fwrite(p, sizeof(double), (size_t)n, f_); }
	void put(const std::string& name, const int* p, int64_t n) { head(name, 'i', n); std::fwrite(p, sizeof(int), (size_t)n, f_); }
	void put(const std::string& name, const std::vector<double>& v) { put(name, v.data(), (int64_t)v.size()); }
	void put(const std::string& name, const std::vector<int>& v) { put(name, v.data(), (int64_t)v.size()); }

private:
	void head(const std::string& name, char kind, int64_t n) {
		int32_t l = (int32_t)name.size();
		std::fwrite(&l, 4, 1, f_);
		std::fwrite(name.data(), 1, name.size(), f_);
		std::fwrite(&kind, 1, 1, f_);
		std::fwrite(&n, 8, 1, f_);
	}
	std::FILE* f_ = nullptr;
};
