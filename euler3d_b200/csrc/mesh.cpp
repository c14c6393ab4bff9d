// Host case model: deck, topology and SU2 block ingest, faces and metrics.
//
// Every formula below reproduces the reference's floating-point expression and
// evaluation order (cited per function) so that the resulting arrays are
// bit-identical to the reference's Block/Cell/Face members.
#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <thread>

namespace e3d {

namespace {

std::string slurp(const std::string& path) {
	std::FILE* f = std::fopen(path.c_str(), "rb");
	if (!f) throw Error(E3D_ERR_IO, "cannot open '" + path + "'");
	std::string s;
	std::fseek(f, 0, SEEK_END);
	long n = std::ftell(f);
	std::fseek(f, 0, SEEK_SET);
	s.resize(n > 0 ? (size_t)n : 0);
	if (n > 0 && std::fread(&s[0], 1, (size_t)n, f) != (size_t)n) {
		std::fclose(f);
		throw Error(E3D_ERR_IO, "short read on '" + path + "'");
	}
	std::fclose(f);
	return s;
}

// Sequential line cursor over a file buffer (the reference reads with getline).
struct Lines {
	const char* p;
	const char* end;
	std::string path;
	long lineno = 0;
	Lines(const std::string& buf, const std::string& file) : p(buf.data()), end(buf.data() + buf.size()), path(file) {}
	// returns [b, e) of the next line without its terminator
	bool next(const char*& b, const char*& e) {
		if (p >= end) return false;
		b = p;
		const char* q = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
		e = q ? q : end;
		p = q ? q + 1 : end;
		++lineno;
		return true;
	}
	void need(const char*& b, const char*& e, const char* what) {
		if (!next(b, e)) fail(std::string("unexpected end of file, expected ") + what);
	}
	[[noreturn]] void fail(const std::string& m) const {
		throw Error(E3D_ERR_FORMAT, path + ":" + std::to_string(lineno) + ": " + m);
	}
};

inline const char* skip_ws(const char* s, const char* e) {
	while (s < e && (*s == ' ' || *s == '\t' || *s == '\r')) ++s;
	return s;
}
inline const char* skip_tok(const char* s, const char* e) {
	while (s < e && !(*s == ' ' || *s == '\t' || *s == '\r')) ++s;
	return s;
}
std::string token(const char*& s, const char* e) {
	s = skip_ws(s, e);
	const char* t = skip_tok(s, e);
	std::string r(s, t);
	s = t;
	return r;
}
bool parse_int(const char*& s, const char* e, long& v) {
	s = skip_ws(s, e);
	if (s >= e) return false;
	char buf[32];
	size_t n = std::min<size_t>((size_t)(skip_tok(s, e) - s), sizeof(buf) - 1);
	std::memcpy(buf, s, n);
	buf[n] = 0;
	char* q;
	v = std::strtol(buf, &q, 10);
	if (q == buf) return false;
	s += (q - buf);
	return true;
}
bool parse_double(const char*& s, const char* e, double& v) {
	s = skip_ws(s, e);
	if (s >= e) return false;
	char buf[64];
	size_t n = std::min<size_t>((size_t)(skip_tok(s, e) - s), sizeof(buf) - 1);
	std::memcpy(buf, s, n);
	buf[n] = 0;
	char* q;
	v = std::strtod(buf, &q);  // same correctly rounded conversion as sscanf("%lf")
	if (q == buf) return false;
	s += (q - buf);
	return true;
}
// "KEYWORD= value" lines, read like sscanf("%s %d")
long keyword_int(Lines& L, const char* what) {
	const char *b, *e;
	L.need(b, e, what);
	token(b, e);
	long v;
	if (!parse_int(b, e, v)) L.fail(std::string("expected ") + what);
	return v;
}

// Local face tables of the reference's face creators: node order fixes the
// stored face node order (FactoryMethod/src/TempTetrahedralFaceCreator.cpp:9,
// TempPrismFaceCreator.cpp:10; SU2 type 12 is the hexahedron there).
const int kTetFaces[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {2, 0, 3}};
const int kHexFaces[6][4] = {{1, 0, 3, 2}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}, {0, 1, 5, 4}, {4, 5, 6, 7}};

struct Key {
	int n[4];
	bool operator<(const Key& o) const {
		for (int k = 0; k < 4; k++)
			if (n[k] != o.n[k]) return n[k] < o.n[k];
		return false;
	}
	bool operator==(const Key& o) const { return n[0] == o.n[0] && n[1] == o.n[1] && n[2] == o.n[2] && n[3] == o.n[3]; }
};
// nn is 3 or 4: face node lists come from the tet/hex face tables and boundary
// elements are read as triangles or quadrilaterals only
Key make_key(const int* nodes, int nn) {
	Key k;
	k.n[3] = -1;
	for (int i = 0; i < nn; i++) k.n[i] = nodes[i];
	for (int i = 1; i < nn; i++)
		for (int j = i; j > 0 && k.n[j - 1] > k.n[j]; j--) std::swap(k.n[j - 1], k.n[j]);
	return k;
}

}  // namespace

// ---------------------------------------------------------------------------
// Deck: the reference reads it with ifstream ignore/getline/>> in a fixed
// sequence (Solver/src/Interface.cpp:35-115); the same stream operations are
// used here so that odd decks parse the same way (e.g. "2.16-16" -> 2.16, -16).
Deck read_deck(const std::string& path) {
	std::ifstream in(path);
	if (!in) throw Error(E3D_ERR_IO, "cannot open deck '" + path + "'");
	Deck d;
	std::string line;
	in.ignore(256, '\n');
	std::getline(in, line);
	in >> d.topology;
	in.ignore(256, '\n');
	in.ignore(256, '\n');
	std::getline(in, line);
	in >> d.cfl >> d.gamma >> d.aoa_deg;
	in.ignore(256, '\n');
	std::getline(in, line);
	in >> d.stages >> d.mach >> d.cmac;
	in.ignore(256, '\n');
	std::getline(in, line);
	in >> d.max_iter >> d.criterion;
	in.ignore(256, '\n');
	std::getline(in, line);
	in >> d.smoothing;
	in.ignore(256, '\n');
	std::getline(in, line);
	in >> d.flux >> d.order;
	in.ignore(256, '\n');
	std::getline(in, line);
	in >> d.gradient >> d.limiter;
	in.ignore(256, '\n');
	std::getline(in, line);
	in >> d.omega >> d.k;
	if (in.fail()) throw Error(E3D_ERR_FORMAT, "deck '" + path + "' is truncated or malformed");
	return d;
}

// ---------------------------------------------------------------------------
// Topology (CompleteMesh.cpp:45-76 for file names, :170-292 for connexions).
Topology read_topology(const std::string& path) {
	std::string buf = slurp(path);
	Lines L(buf, path);
	Topology t;
	const long nb = keyword_int(L, "NBLOCK=");
	if (nb <= 0 || nb > (1 << 20)) L.fail("bad NBLOCK");
	for (long i = 0; i < nb; i++) {
		const char *b, *e;
		L.need(b, e, "block file name");
		std::string name = token(b, e);
		if (name.empty()) L.fail("empty block file name");
		t.block_files.push_back(name);
	}
	struct Entry {
		long ghost_count = 0;
		std::vector<std::pair<long, std::vector<int>>> marks;
		bool present = false;
	};
	std::vector<Entry> entries((size_t)nb);
	for (long i = 0; i < nb; i++) {
		const char *b, *e;
		if (!L.next(b, e)) break;  // trailing entries may be absent: no connexions
		token(b, e);
		long idx;
		if (!parse_int(b, e, idx) || idx < 0 || idx >= nb) L.fail("bad Block= line");
		Entry& en = entries[(size_t)idx];
		en.present = true;
		en.ghost_count = keyword_int(L, "GhostCount=");
		const long m = keyword_int(L, "Nconnexion=");
		for (long j = 0; j < m; j++) {
			const long origin = keyword_int(L, "Nmark=");
			const long k = keyword_int(L, "Nelems=");
			if (origin < 0 || origin >= nb || k < 0) L.fail("bad connexion header");
			std::vector<int> cells((size_t)k);
			for (long q = 0; q < k; q++) {
				const char *cb, *ce;
				L.need(cb, ce, "connexion cell id");
				long v;
				if (!parse_int(cb, ce, v)) L.fail("bad connexion cell id");
				cells[(size_t)q] = (int)v;
			}
			en.marks.emplace_back(origin, std::move(cells));
		}
	}
	for (long blk = 0; blk < nb; blk++) {
		const Entry& en = entries[(size_t)blk];
		long count = en.ghost_count;
		for (const auto& mk : en.marks) {
			Connexion c;
			c.dest_block = (int)blk;
			c.origin_block = (int)mk.first;
			c.origin_cells = mk.second;
			c.dest_cells.resize(mk.second.size());
			for (size_t q = 0; q < mk.second.size(); q++) c.dest_cells[q] = (int)(count++);
			t.connexions.push_back(std::move(c));
		}
	}
	return t;
}

// ---------------------------------------------------------------------------
// SU2 block reader (ConcreteBlockBuilder.cpp:22-225 counts, :227-495 reads).
HostBlock load_block(const std::string& path, int block_id) {
	std::string buf = slurp(path);
	Lines L(buf, path);
	HostBlock B;
	B.id = block_id;
	const char *b, *e;
	L.need(b, e, "NDIME=");
	L.need(b, e, "blank line");
	const long n_nodes = keyword_int(L, "NPOIN=");
	if (n_nodes <= 0 || n_nodes > (1L << 30)) L.fail("bad NPOIN");
	B.n_nodes = (int)n_nodes;
	B.node_xyz.resize(3 * (size_t)n_nodes);
	for (long i = 0; i < n_nodes; i++) {
		L.need(b, e, "node coordinates");
		for (int k = 0; k < 3; k++)
			if (!parse_double(b, e, B.node_xyz[3 * (size_t)i + k])) L.fail("bad node coordinate");
	}
	L.need(b, e, "blank line");
	const long n_real = keyword_int(L, "NELEM=");
	if (n_real <= 0 || n_real > (1L << 30)) L.fail("bad NELEM");
	B.n_real = (int)n_real;
	B.cell_type.resize((size_t)n_real);
	B.cell_node_ptr.assign(1, 0);
	B.cell_nodes.reserve((size_t)n_real * 4);
	for (long i = 0; i < n_real; i++) {
		L.need(b, e, "element");
		long type;
		if (!parse_int(b, e, type)) L.fail("bad element type");
		int nn;
		if (type == 10) nn = 4;
		else if (type == 12) nn = 8;
		else if (type == 14)
			L.fail("pyramids (type 14) are not supported: the reference's pyramid face table is released "
			       "before use (FactoryMethod/src/TempPyramidFaceCreator.cpp:59-65)");
		else L.fail("unsupported element type " + std::to_string(type));
		B.cell_type[(size_t)i] = (int)type;
		for (int k = 0; k < nn; k++) {
			long v;
			if (!parse_int(b, e, v)) L.fail("bad element node id");
			if (v < 0 || v >= n_nodes) L.fail("element node id out of range");
			B.cell_nodes.push_back((int)v);
		}
		B.cell_node_ptr.push_back((int)B.cell_nodes.size());
	}
	L.need(b, e, "blank line");
	const long n_mark = keyword_int(L, "NMARK=");
	if (n_mark < 0 || n_mark > 100000) L.fail("bad NMARK");
	int cell_id = (int)n_real;
	int n_connexion = 0;
	for (long m = 0; m < n_mark; m++) {
		L.need(b, e, "MARKER_TAG=");
		token(b, e);
		std::string tag = token(b, e);
		Marker mk;
		if (tag == "WALL") mk.kind = MK_WALL;
		else if (tag == "FARFIELD") mk.kind = MK_FARFIELD;
		else if (tag == "SYMMETRY") mk.kind = MK_SYMMETRY;
		else if (tag == "CONNEXION") { mk.kind = MK_CONNEXION; n_connexion++; }
		else L.fail("unknown marker '" + tag + "'");
		const long k = keyword_int(L, "MARKER_ELEMS=");
		if (k < 0 || k > (1L << 30)) L.fail("bad MARKER_ELEMS");
		for (long q = 0; q < k; q++) {
			L.need(b, e, "boundary element");
			long type;
			if (!parse_int(b, e, type)) L.fail("bad boundary element type");
			int nn;
			if (type == 5) nn = 3;
			else if (type == 9) nn = 4;
			else L.fail("unsupported boundary element type " + std::to_string(type));
			for (int j = 0; j < nn; j++) {
				long v;
				if (!parse_int(b, e, v)) L.fail("bad boundary node id");
				if (v < 0 || v >= n_nodes) L.fail("boundary node id out of range");
				B.cell_nodes.push_back((int)v);
			}
			B.cell_node_ptr.push_back((int)B.cell_nodes.size());
			mk.ghosts.push_back(cell_id++);
		}
		B.markers.push_back(std::move(mk));
	}
	B.n_all = cell_id;
	// ConcreteBlockBuilder.cpp:107-108,143-149: BCs apply to the first
	// (n_markers - n_connexion_markers) markers, whatever their kind.
	B.n_real_boundaries = (int)n_mark - n_connexion;
	finish_block(B);
	return B;
}

// ---------------------------------------------------------------------------
void finish_block(HostBlock& B) {
	const int nr = B.n_real, na = B.n_all;
	// ---- faces in first-occurrence order (ConcreteBlockBuilder.cpp:541-738) ----
	std::vector<int> cand_ptr(1, 0);
	for (int c = 0; c < nr; c++) cand_ptr.push_back(cand_ptr.back() + (B.cell_type[c] == 12 ? 6 : 4));
	const size_t Q = (size_t)cand_ptr.back();
	std::vector<Key> keys(Q);
	std::vector<int> cand_nodes(Q * 4, -1), cand_nn(Q), cand_cell(Q);
	for (int c = 0; c < nr; c++) {
		const int* cn = &B.cell_nodes[B.cell_node_ptr[c]];
		const bool hex = B.cell_type[c] == 12;
		const int nf = hex ? 6 : 4, nn = hex ? 4 : 3;
		for (int j = 0; j < nf; j++) {
			const size_t q = (size_t)cand_ptr[c] + j;
			for (int k = 0; k < nn; k++) cand_nodes[q * 4 + k] = cn[hex ? kHexFaces[j][k] : kTetFaces[j][k]];
			cand_nn[q] = nn;
			cand_cell[q] = c;
			keys[q] = make_key(&cand_nodes[q * 4], nn);
		}
	}
	std::vector<uint32_t> order(Q);
	std::iota(order.begin(), order.end(), 0u);
	std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
		if (keys[a] == keys[b]) return a < b;
		return keys[a] < keys[b];
	});
	std::vector<int> creator_of(Q, -1);  // candidate -> creating candidate
	std::vector<int> partner_cell(Q, -1);  // creator candidate -> other cell
	std::vector<char> is_creator(Q, 0);
	for (size_t i = 0; i < Q;) {
		size_t j = i + 1;
		while (j < Q && keys[order[j]] == keys[order[i]]) j++;
		const uint32_t cr = order[i];
		if (j - i > 2) throw Error(E3D_ERR_MESH, "block " + std::to_string(B.id) + ": face shared by more than two cells");
		is_creator[cr] = 1;
		for (size_t t = i; t < j; t++) creator_of[order[t]] = (int)cr;
		if (j - i == 2) {
			if (cand_cell[order[i + 1]] == cand_cell[cr])
				throw Error(E3D_ERR_MESH, "block " + std::to_string(B.id) + ": degenerate cell with a repeated face");
			partner_cell[cr] = cand_cell[order[i + 1]];
		}
		i = j;
	}
	std::vector<int> face_of_creator(Q, -1);
	int nf = 0;
	for (size_t q = 0; q < Q; q++)
		if (is_creator[q]) face_of_creator[q] = nf++;
	B.n_faces = nf;
	B.face_nnodes.resize(nf);
	B.face_node_ptr.assign(1, 0);
	B.face_cells.assign(2 * (size_t)nf, -1);
	{
		std::vector<int> first(nf), second(nf, -1);
		for (size_t q = 0; q < Q; q++) {
			if (!is_creator[q]) continue;
			const int f = face_of_creator[q];
			B.face_nnodes[f] = cand_nn[q];
			for (int k = 0; k < cand_nn[q]; k++) B.face_nodes.push_back(cand_nodes[q * 4 + k]);
			B.face_node_ptr.push_back((int)B.face_nodes.size());
			first[f] = cand_cell[q];
			second[f] = partner_cell[q];
		}
		// ghost cells close boundary faces (the reference finds the two cells
		// through shared nodes, BlockBuilder.cpp:248-334; left = lower id)
		for (int g = nr; g < na; g++) {
			const int nn = B.cell_node_ptr[g + 1] - B.cell_node_ptr[g];
			Key k = make_key(&B.cell_nodes[B.cell_node_ptr[g]], nn);
			auto it = std::lower_bound(order.begin(), order.end(), k,
			                           [&](uint32_t a, const Key& kk) { return keys[a] < kk; });
			if (it == order.end() || !(keys[*it] == k))
				throw Error(E3D_ERR_MESH, "block " + std::to_string(B.id) + ": boundary element " +
				                              std::to_string(g) + " matches no cell face");
			const int f = face_of_creator[creator_of[*it]];
			if (second[f] != -1)
				throw Error(E3D_ERR_MESH, "block " + std::to_string(B.id) + ": boundary element " +
				                              std::to_string(g) + " lies on an interior or already closed face");
			second[f] = g;
		}
		for (int f = 0; f < nf; f++) {
			if (second[f] < 0)
				throw Error(E3D_ERR_MESH, "block " + std::to_string(B.id) + ": face " + std::to_string(f) +
				                              " has one cell and no boundary marker element");
			B.face_cells[2 * (size_t)f] = std::min(first[f], second[f]);
			B.face_cells[2 * (size_t)f + 1] = std::max(first[f], second[f]);
		}
	}
	// ---- cell -> faces / cells in ascending face id (BlockBuilder.cpp:355-377) ----
	B.cell_face_ptr.assign((size_t)na + 1, 0);
	for (int c = 0; c < na; c++)
		B.cell_face_ptr[c + 1] = B.cell_face_ptr[c] + (c < nr ? (B.cell_type[c] == 12 ? 6 : 4) : 1);
	B.cell_faces.assign((size_t)B.cell_face_ptr[na], -1);
	B.cell_cells.assign((size_t)B.cell_face_ptr[na], -1);
	{
		std::vector<int> fill(na, 0);
		for (int f = 0; f < nf; f++) {
			const int l = B.face_cells[2 * (size_t)f], r = B.face_cells[2 * (size_t)f + 1];
			if (fill[l] >= B.cell_face_ptr[l + 1] - B.cell_face_ptr[l] || fill[r] >= B.cell_face_ptr[r + 1] - B.cell_face_ptr[r])
				throw Error(E3D_ERR_MESH, "block " + std::to_string(B.id) + ": cell face count overflow");
			B.cell_faces[B.cell_face_ptr[l] + fill[l]] = f;
			B.cell_cells[B.cell_face_ptr[l] + fill[l]++] = r;
			B.cell_faces[B.cell_face_ptr[r] + fill[r]] = f;
			B.cell_cells[B.cell_face_ptr[r] + fill[r]++] = l;
		}
		for (int c = 0; c < na; c++)
			if (fill[c] != B.cell_face_ptr[c + 1] - B.cell_face_ptr[c])
				throw Error(E3D_ERR_MESH, "block " + std::to_string(B.id) + ": cell " + std::to_string(c) + " is not closed");
	}
	// wall face ids (BlockBuilder.cpp:382-395): WALL ghosts in marker order
	B.wall_faces.clear();
	for (const Marker& m : B.markers)
		if (m.kind == MK_WALL)
			for (int g : m.ghosts) B.wall_faces.push_back(B.cell_faces[B.cell_face_ptr[g]]);

	// ---- metrics (Metrics/src/MetricsInitializer.cpp:27-54 call order) ----
	const double* X = B.node_xyz.data();
	B.cell_center.assign(3 * (size_t)na, 0.0);
	// computeCenterCells (:57-107): node mean; ghosts copy their interior cell
	for (int c = 0; c < nr; c++) {
		double sx = 0.0, sy = 0.0, sz = 0.0;
		const int n = B.cell_node_ptr[c + 1] - B.cell_node_ptr[c];
		for (int j = 0; j < n; j++) {
			const int v = B.cell_nodes[B.cell_node_ptr[c] + j];
			sx += X[3 * (size_t)v];
			sy += X[3 * (size_t)v + 1];
			sz += X[3 * (size_t)v + 2];
		}
		B.cell_center[3 * (size_t)c] = sx / n;
		B.cell_center[3 * (size_t)c + 1] = sy / n;
		B.cell_center[3 * (size_t)c + 2] = sz / n;
	}
	for (int g = nr; g < na; g++) {
		const int in = B.cell_cells[B.cell_face_ptr[g]];
		for (int k = 0; k < 3; k++) B.cell_center[3 * (size_t)g + k] = B.cell_center[3 * (size_t)in + k];
	}
	// computeCenterFaces (:109-143)
	B.face_center.assign(3 * (size_t)nf, 0.0);
	for (int f = 0; f < nf; f++) {
		double sx = 0.0, sy = 0.0, sz = 0.0;
		const int n = B.face_nnodes[f];
		for (int j = 0; j < n; j++) {
			const int v = B.face_nodes[B.face_node_ptr[f] + j];
			sx += X[3 * (size_t)v];
			sy += X[3 * (size_t)v + 1];
			sz += X[3 * (size_t)v + 2];
		}
		B.face_center[3 * (size_t)f] = sx / n;
		B.face_center[3 * (size_t)f + 1] = sy / n;
		B.face_center[3 * (size_t)f + 2] = sz / n;
	}
	// computeNormalFaces (:308-449): triangle shoelace / quad diagonals, then
	// flipped to point away from the left cell centre
	B.face_normal.assign(3 * (size_t)nf, 0.0);
	for (int f = 0; f < nf; f++) {
		const int* fn = &B.face_nodes[B.face_node_ptr[f]];
		double sx, sy, sz;
		if (B.face_nnodes[f] == 3) {
			const double x1 = X[3 * (size_t)fn[0]], y1 = X[3 * (size_t)fn[0] + 1], z1 = X[3 * (size_t)fn[0] + 2];
			const double x2 = X[3 * (size_t)fn[1]], y2 = X[3 * (size_t)fn[1] + 1], z2 = X[3 * (size_t)fn[1] + 2];
			const double x3 = X[3 * (size_t)fn[2]], y3 = X[3 * (size_t)fn[2] + 1], z3 = X[3 * (size_t)fn[2] + 2];
			const double dxyA = (x1 - x2) * (y1 + y2), dxyB = (x2 - x3) * (y2 + y3), dxyC = (x3 - x1) * (y3 + y1);
			const double dyzA = (y1 - y2) * (z1 + z2), dyzB = (y2 - y3) * (z2 + z3), dyzC = (y3 - y1) * (z3 + z1);
			const double dzxA = (z1 - z2) * (x1 + x2), dzxB = (z2 - z3) * (x2 + x3), dzxC = (z3 - z1) * (x3 + x1);
			sx = 0.5 * (dyzA + dyzB + dyzC);
			sy = 0.5 * (dzxA + dzxB + dzxC);
			sz = 0.5 * (dxyA + dxyB + dxyC);
		} else {
			const double x1 = X[3 * (size_t)fn[0]], y1 = X[3 * (size_t)fn[0] + 1], z1 = X[3 * (size_t)fn[0] + 2];
			const double x2 = X[3 * (size_t)fn[1]], y2 = X[3 * (size_t)fn[1] + 1], z2 = X[3 * (size_t)fn[1] + 2];
			const double x3 = X[3 * (size_t)fn[2]], y3 = X[3 * (size_t)fn[2] + 1], z3 = X[3 * (size_t)fn[2] + 2];
			const double x4 = X[3 * (size_t)fn[3]], y4 = X[3 * (size_t)fn[3] + 1], z4 = X[3 * (size_t)fn[3] + 2];
			const double dxA = x4 - x2, dxB = x3 - x1, dyA = y4 - y2, dyB = y3 - y1, dzA = z4 - z2, dzB = z3 - z1;
			sx = 0.5 * (dyA * dzB - dzA * dyB);
			sy = 0.5 * (dzA * dxB - dxA * dzB);
			sz = 0.5 * (dxA * dyB - dyA * dxB);
		}
		const int l = B.face_cells[2 * (size_t)f];
		const double cx = B.face_center[3 * (size_t)f] - B.cell_center[3 * (size_t)l];
		const double cy = B.face_center[3 * (size_t)f + 1] - B.cell_center[3 * (size_t)l + 1];
		const double cz = B.face_center[3 * (size_t)f + 2] - B.cell_center[3 * (size_t)l + 2];
		const double dot = cx * sx + cy * sy + cz * sz;
		if (dot < 0) {
			sx *= -1.0;
			sy *= -1.0;
			sz *= -1.0;
		}
		B.face_normal[3 * (size_t)f] = sx;
		B.face_normal[3 * (size_t)f + 1] = sy;
		B.face_normal[3 * (size_t)f + 2] = sz;
	}
	// computeAreaFaces (:546-562)
	B.face_area.resize(nf);
	for (int f = 0; f < nf; f++) {
		const double sx = B.face_normal[3 * (size_t)f], sy = B.face_normal[3 * (size_t)f + 1], sz = B.face_normal[3 * (size_t)f + 2];
		B.face_area[f] = std::sqrt(sx * sx + sy * sy + sz * sz);
	}
	// computeVolumeCells (:565-638): divergence theorem with outward normals
	B.cell_volume.assign((size_t)na, 0.0);
	for (int c = 0; c < nr; c++) {
		double vol = 0.0;
		for (int s = B.cell_face_ptr[c]; s < B.cell_face_ptr[c + 1]; s++) {
			const int f = B.cell_faces[s];
			const double fx = B.face_center[3 * (size_t)f], fy = B.face_center[3 * (size_t)f + 1], fz = B.face_center[3 * (size_t)f + 2];
			double sx = B.face_normal[3 * (size_t)f], sy = B.face_normal[3 * (size_t)f + 1], sz = B.face_normal[3 * (size_t)f + 2];
			const double c0 = fx - B.cell_center[3 * (size_t)c], c1 = fy - B.cell_center[3 * (size_t)c + 1],
			             c2 = fz - B.cell_center[3 * (size_t)c + 2];
			const double dot = c0 * sx + c1 * sy + c2 * sz;
			if (dot < 0) {
				sx *= -1.0;
				sy *= -1.0;
				sz *= -1.0;
			}
			vol += (fx * sx + fy * sy + fz * sz) / 3;
		}
		B.cell_volume[c] = vol;
	}
	for (int g = nr; g < na; g++) B.cell_volume[g] = B.cell_volume[B.cell_cells[B.cell_face_ptr[g]]];
	// computeInterpVect (:451-543): r = face centre - cell centre; the ghost
	// side is the left vector reflected about the face plane
	B.r_left.assign(3 * (size_t)nf, 0.0);
	B.r_right.assign(3 * (size_t)nf, 0.0);
	for (int f = 0; f < nf; f++) {
		const int l = B.face_cells[2 * (size_t)f], r = B.face_cells[2 * (size_t)f + 1];
		for (int k = 0; k < 3; k++) {
			B.r_left[3 * (size_t)f + k] = B.face_center[3 * (size_t)f + k] - B.cell_center[3 * (size_t)l + k];
			B.r_right[3 * (size_t)f + k] = B.face_center[3 * (size_t)f + k] - B.cell_center[3 * (size_t)r + k];
		}
	}
	for (int g = nr; g < na; g++) {
		const int f = B.cell_faces[B.cell_face_ptr[g]];
		const double rx = B.r_left[3 * (size_t)f], ry = B.r_left[3 * (size_t)f + 1], rz = B.r_left[3 * (size_t)f + 2];
		const double area = B.face_area[f];
		const double nx = B.face_normal[3 * (size_t)f] / area, ny = B.face_normal[3 * (size_t)f + 1] / area,
		             nz = B.face_normal[3 * (size_t)f + 2] / area;
		const double p = rx * nx + ry * ny + rz * nz;
		B.r_right[3 * (size_t)f] = rx - 2 * p * nx;
		B.r_right[3 * (size_t)f + 1] = ry - 2 * p * ny;
		B.r_right[3 * (size_t)f + 2] = rz - 2 * p * nz;
	}
	// computeCenterGhostCells (:640-671): mirror the interior centre through the face
	for (int g = nr; g < na; g++) {
		const int f = B.cell_faces[B.cell_face_ptr[g]];
		for (int k = 0; k < 3; k++) B.cell_center[3 * (size_t)g + k] += 2.0 * B.r_left[3 * (size_t)f + k];
	}
	// computeWLS (:673-800): unweighted least squares by Gram-Schmidt (QR)
	B.ls_weights.assign(3 * (size_t)B.cell_face_ptr[nr], 0.0);
	if (nr > 1) {
		std::vector<double> dx, dy, dz;
		for (int c = 0; c < nr; c++) {
			const int s0 = B.cell_face_ptr[c], n = B.cell_face_ptr[c + 1] - s0;
			dx.resize(n);
			dy.resize(n);
			dz.resize(n);
			for (int j = 0; j < n; j++) {
				const int nb = B.cell_cells[s0 + j];
				dx[j] = B.cell_center[3 * (size_t)nb] - B.cell_center[3 * (size_t)c];
				dy[j] = B.cell_center[3 * (size_t)nb + 1] - B.cell_center[3 * (size_t)c + 1];
				dz[j] = B.cell_center[3 * (size_t)nb + 2] - B.cell_center[3 * (size_t)c + 2];
			}
			double sxx = 0.0, sxy = 0.0, sxz = 0.0, syy = 0.0, syz = 0.0, szz = 0.0;
			for (int j = 0; j < n; j++) {
				sxx += dx[j] * dx[j];
				sxy += dx[j] * dy[j];
				sxz += dx[j] * dz[j];
			}
			const double r11 = std::sqrt(sxx);
			const double r12 = (1 / r11) * sxy;
			const double r13 = (1 / r11) * sxz;
			for (int j = 0; j < n; j++) {
				syy += dy[j] * dy[j];
				syz += dy[j] * dz[j];
			}
			const double r22 = std::sqrt(syy - r12 * r12);
			const double r23 = (1 / r22) * (syz - r12 * r13);
			for (int j = 0; j < n; j++) szz += dz[j] * dz[j];
			const double r33 = std::sqrt(szz - (r13 * r13 + r23 * r23));
			const double beta = (r12 * r23 - r13 * r22) / (r11 * r22);
			for (int j = 0; j < n; j++) {
				const double a3 = (1 / (r33 * r33)) * (dz[j] - (r23 / r22) * dy[j] + beta * dx[j]);
				const double a2 = (1 / (r22 * r22)) * (dy[j] - (r12 / r11) * dx[j]);
				const double a1 = dx[j] / (r11 * r11);
				double* w = &B.ls_weights[3 * (size_t)(s0 + j)];
				w[0] = a1 - (r12 / r11) * a2 + beta * a3;
				w[1] = a2 - (r23 / r22) * a3;
				w[2] = a3;
			}
		}
	}
}

// ---------------------------------------------------------------------------
HostCase load_case(const std::string& deck_path, const std::string& workdir, int n_threads) {
	auto resolve = [&](const std::string& p) {
		if (p.empty() || p[0] == '/' || workdir.empty()) return p;
		return workdir + "/" + p;
	};
	HostCase hc;
	hc.deck = read_deck(deck_path);
	hc.topo = read_topology(resolve(hc.deck.topology));
	const int nb = (int)hc.topo.block_files.size();
	hc.blocks.resize(nb);
	if (n_threads <= 0) n_threads = (int)std::max(1u, std::thread::hardware_concurrency());
	n_threads = std::min(n_threads, nb);
	std::vector<std::string> errors(nb);
	std::vector<int> codes(nb, 0);
	auto work = [&](int t) {
		for (int b = t; b < nb; b += n_threads) {
			try {
				hc.blocks[b] = load_block(resolve(hc.topo.block_files[b]), b);
			} catch (const Error& e) {
				codes[b] = e.code;
				errors[b] = e.what();
			} catch (const std::exception& e) {
				codes[b] = E3D_ERR_MESH;
				errors[b] = e.what();
			}
		}
	};
	std::vector<std::thread> pool;
	for (int t = 1; t < n_threads; t++) pool.emplace_back(work, t);
	work(0);
	for (auto& th : pool) th.join();
	for (int b = 0; b < nb; b++)
		if (codes[b]) throw Error(codes[b], errors[b]);
	// every connexion index must be inside its blocks before anything reaches a device
	for (const Connexion& c : hc.topo.connexions) {
		const HostBlock& d = hc.blocks[c.dest_block];
		const HostBlock& o = hc.blocks[c.origin_block];
		for (size_t q = 0; q < c.dest_cells.size(); q++) {
			if (c.dest_cells[q] < d.n_real || c.dest_cells[q] >= d.n_all)
				throw Error(E3D_ERR_MESH, "topology: connexion ghost " + std::to_string(c.dest_cells[q]) +
				                              " outside the ghost range of block " + std::to_string(c.dest_block));
			if (c.origin_cells[q] < 0 || c.origin_cells[q] >= o.n_all)
				throw Error(E3D_ERR_MESH, "topology: origin cell " + std::to_string(c.origin_cells[q]) +
				                              " outside block " + std::to_string(c.origin_block));
		}
	}
	return hc;
}

}  // namespace e3d
