// Device order of the real cells of a block.
//
// The reference keeps cells in file order (ConcreteBlockBuilder.cpp:289-368
// numbers them as the SU2 file lists them).  On the GPU the order decides how
// well neighbour gathers share cache lines: a thread block works on 128
// consecutive cells and reads the states of their neighbours, so cells that
// are close in the mesh should be close in memory.  Renumbering changes only
// where a cell's data sits on the device: a cell's slots keep its ascending
// face id order, faces keep their ids and orientation, so every per-cell sum
// runs in the reference's order and FP64 results stay bit for bit the same.
//
//   RENUMBER_RCM      reverse Cuthill-McKee on the real-cell adjacency graph
//                     (breadth-first levels from a pseudo-peripheral cell,
//                     neighbours by ascending degree, the whole order reversed)
//   RENUMBER_MORTON   Z-order of the cell centres (21 bits per axis over the
//                     block's bounding box, one scale for all three axes)
//   RENUMBER_SHUFFLE  a seeded random order: the worst case, for tests and
//                     measurement
//
// RENUMBER_BOUNDARY_LAST, added to any of these, then moves the cells that
// have a ghost neighbour (a boundary or connexion face) to the end of the
// block, each group keeping the base order.  The stage passes do extra work
// for such a cell (the ghost's reflected gradient, limiter and face state;
// its boundary condition); a warp runs that work if any of its 32 cells needs
// it, and in file order nearly every warp holds one.  Grouped, only the
// boundary cells' warps run it.
#include <algorithm>
#include <cstdint>
#include <numeric>

#include "engine.hpp"

namespace e3d {
namespace {

// neighbours of real cell c that are real cells, in slot order
template <class F>
void for_real_neighbours(const HostBlock& b, int c, F&& f) {
	for (int j = b.cell_face_ptr[c]; j < b.cell_face_ptr[c + 1]; j++) {
		const int nb = b.cell_cells[j];
		if (nb < b.n_real) f(nb);
	}
}

// Breadth-first levels from `start` over unvisited cells; returns the cells of
// the last level (eccentricity = number of levels - 1 in *depth).
std::vector<int> last_level(const HostBlock& b, int start, const std::vector<char>& visited, std::vector<int>& mark,
                            int stamp, int* depth) {
	std::vector<int> cur{start}, next;
	mark[start] = stamp;
	int d = 0;
	while (true) {
		next.clear();
		for (int c : cur)
			for_real_neighbours(b, c, [&](int nb) {
				if (!visited[nb] && mark[nb] != stamp) {
					mark[nb] = stamp;
					next.push_back(nb);
				}
			});
		if (next.empty()) break;
		cur.swap(next);
		d++;
	}
	*depth = d;
	return cur;
}

std::vector<int> rcm(const HostBlock& b) {
	const int n = b.n_real;
	std::vector<int> deg(n, 0);
	for (int c = 0; c < n; c++) for_real_neighbours(b, c, [&](int) { deg[c]++; });
	std::vector<int> by_degree(n);
	std::iota(by_degree.begin(), by_degree.end(), 0);
	std::stable_sort(by_degree.begin(), by_degree.end(), [&](int x, int y) { return deg[x] < deg[y]; });
	std::vector<char> visited(n, 0);
	std::vector<int> mark(n, -1), order;
	order.reserve(n);
	int stamp = 0;
	size_t pick = 0;
	while ((int)order.size() < n) {
		while (visited[by_degree[pick]]) pick++;
		// pseudo-peripheral start (George-Liu): move to a least-degree cell of the
		// last level while the eccentricity grows
		int start = by_degree[pick], depth = 0;
		std::vector<int> last = last_level(b, start, visited, mark, stamp++, &depth);
		for (int tries = 0; tries < 8; tries++) {
			const int cand = *std::min_element(last.begin(), last.end(), [&](int x, int y) {
				return deg[x] < deg[y] || (deg[x] == deg[y] && x < y);
			});
			int d2 = 0;
			std::vector<int> l2 = last_level(b, cand, visited, mark, stamp++, &d2);
			if (d2 <= depth) break;
			start = cand;
			depth = d2;
			last.swap(l2);
		}
		// Cuthill-McKee levels: unvisited neighbours by ascending degree, then id
		const size_t first = order.size();
		order.push_back(start);
		visited[start] = 1;
		std::vector<int> nbs;
		for (size_t h = first; h < order.size(); h++) {
			nbs.clear();
			for_real_neighbours(b, order[h], [&](int nb) {
				if (!visited[nb]) {
					visited[nb] = 1;
					nbs.push_back(nb);
				}
			});
			std::sort(nbs.begin(), nbs.end(), [&](int x, int y) { return deg[x] < deg[y] || (deg[x] == deg[y] && x < y); });
			order.insert(order.end(), nbs.begin(), nbs.end());
		}
	}
	std::reverse(order.begin(), order.end());
	return order;
}

uint64_t spread21(uint64_t v) {  // bits of a 21-bit value, two zeros between each
	v &= 0x1fffff;
	v = (v | v << 32) & 0x1f00000000ffffULL;
	v = (v | v << 16) & 0x1f0000ff0000ffULL;
	v = (v | v << 8) & 0x100f00f00f00f00fULL;
	v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
	v = (v | v << 2) & 0x1249249249249249ULL;
	return v;
}

std::vector<int> morton(const HostBlock& b) {
	const int n = b.n_real;
	double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
	for (int c = 0; c < n; c++)
		for (int d = 0; d < 3; d++) {
			lo[d] = std::min(lo[d], b.cell_center[3 * (size_t)c + d]);
			hi[d] = std::max(hi[d], b.cell_center[3 * (size_t)c + d]);
		}
	const double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
	const double scale = 2097151.0 / ext;
	std::vector<uint64_t> key(n);
	for (int c = 0; c < n; c++) {
		uint64_t k = 0;
		for (int d = 0; d < 3; d++) {
			const double x = (b.cell_center[3 * (size_t)c + d] - lo[d]) * scale;
			const uint64_t q = (uint64_t)std::min(2097151.0, std::max(0.0, x));
			k |= spread21(q) << d;
		}
		key[c] = k;
	}
	std::vector<int> order(n);
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key[x] < key[y]; });
	return order;
}

uint64_t splitmix64(uint64_t& s) {
	uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
	return z ^ (z >> 31);
}

std::vector<int> shuffled(const HostBlock& b) {
	std::vector<int> order(b.n_real);
	std::iota(order.begin(), order.end(), 0);
	uint64_t s = 0x5eed0000ULL + (uint64_t)b.id;
	for (int i = b.n_real - 1; i > 0; i--) std::swap(order[i], order[splitmix64(s) % (uint64_t)(i + 1)]);
	return order;
}


std::vector<int> base_order(const HostBlock& b, int mode) {
	switch (mode) {
	case RENUMBER_NONE: {
		std::vector<int> order(b.n_real);
		std::iota(order.begin(), order.end(), 0);
		return order;
	}
	case RENUMBER_RCM: return rcm(b);
	case RENUMBER_MORTON: return morton(b);
	case RENUMBER_SHUFFLE: return shuffled(b);
	default: throw Error(E3D_ERR_ARG, "unknown cell renumbering " + std::to_string(mode));
	}
}

}  // namespace

std::vector<int> cell_order(const HostBlock& b, int mode) {
	if (mode < 0 || (mode & ~(RENUMBER_BOUNDARY_LAST | 15)) != 0)
		throw Error(E3D_ERR_ARG, "unknown cell renumbering " + std::to_string(mode));
	std::vector<int> order = base_order(b, mode & 15);
	if (mode & RENUMBER_BOUNDARY_LAST) {
		std::vector<char> boundary(b.n_real, 0);
		for (int c = 0; c < b.n_real; c++)
			for (int j = b.cell_face_ptr[c]; j < b.cell_face_ptr[c + 1]; j++)
				if (b.cell_cells[j] >= b.n_real) boundary[c] = 1;
		std::stable_partition(order.begin(), order.end(), [&](int c) { return !boundary[c]; });
	}
	return order;
}

}  // namespace e3d
