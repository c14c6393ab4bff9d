// Host-side case model: input deck, topology, SU2 blocks, faces and metrics.
//
// This is the host input boundary of the residual/update path.  It reads the
// same three files as the reference program and produces, per block, the
// arrays the reference keeps in its Block/Cell/Face objects, with the same cell
// numbering, face numbering, face orientation and metric values (bit for bit),
// so that device kernels summing in the reference's order reproduce its results.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/e3d.h"

namespace e3d {

struct Error : std::runtime_error {
	int code;
	Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Status codes are the C ABI's E3D_* values (include/e3d.h).

// Positional input deck (reference Solver/src/Interface.cpp:14-237).
struct Deck {
	std::string topology;
	double cfl = 1.5, gamma = 1.4, aoa_deg = 0.0;
	int stages = 5;
	double mach = 0.5, cmac = 1.0;
	int max_iter = 1;
	double criterion = -15.0;
	bool smoothing = false;
	std::string flux = "roe";
	int order = 1;
	std::string gradient = "leastsquares";
	std::string limiter = "venkatakrishnan";
	double omega = 0.0, k = 5.0;
};
Deck read_deck(const std::string& path);

enum MarkerKind : int { MK_WALL = 1, MK_FARFIELD = 2, MK_SYMMETRY = 3, MK_CONNEXION = 4 };

struct Marker {
	int kind;
	std::vector<int> ghosts;  // block-local ghost cell ids, in file order
};

// One inter-block copy list (reference ConnexionCellIds, CompleteMesh.cpp:218-257).
struct Connexion {
	int dest_block, origin_block;
	std::vector<int> dest_cells;    // ghost cells of dest_block
	std::vector<int> origin_cells;  // cells of origin_block
};

struct Topology {
	std::vector<std::string> block_files;
	std::vector<Connexion> connexions;  // in reference registration order
};
Topology read_topology(const std::string& path);

// One block with the reference's per-object data flattened into arrays.
struct HostBlock {
	int id = 0;
	int n_real = 0, n_all = 0, n_faces = 0, n_nodes = 0;
	int n_real_boundaries = 0;  // markers [0, n_real_boundaries) get BC updates
	std::vector<double> node_xyz;               // 3*n_nodes
	std::vector<int> cell_type;                 // SU2 type per real cell (10, 12, 14)
	std::vector<int> cell_node_ptr, cell_nodes;  // CSR over all cells (ghosts: 3 or 4 nodes)
	std::vector<Marker> markers;
	// faces
	std::vector<int> face_nnodes, face_node_ptr, face_nodes;
	std::vector<int> face_cells;    // 2*n_faces: left (lower id), right
	std::vector<double> face_normal;  // 3*n_faces area vector oriented left -> right
	std::vector<double> face_area;    // n_faces
	std::vector<double> face_center;  // 3*n_faces
	std::vector<double> r_left, r_right;  // 3*n_faces
	// cells
	std::vector<int> cell_face_ptr;  // n_all+1
	std::vector<int> cell_faces;     // ascending face id
	std::vector<int> cell_cells;     // neighbour across the same face
	std::vector<double> cell_volume;  // n_all
	std::vector<double> cell_center;  // 3*n_all
	std::vector<double> ls_weights;   // 3 per real-cell slot (cell_face_ptr order)
	std::vector<int> wall_faces;      // faces of WALL markers in marker order
};

// Reads one SU2-dialect block (ConcreteBlockBuilder.cpp:22-495), builds faces
// (:497-742, first-occurrence order), connectivity (BlockBuilder.cpp:147-458)
// and metrics (Metrics/src/MetricsInitializer.cpp:27-800).
HostBlock load_block(const std::string& path, int block_id);

// Builds faces, connectivity and metrics for a block whose nodes, cells and
// markers are already filled (used by load_block and by in-memory callers).
void finish_block(HostBlock& b);

struct HostCase {
	Deck deck;
	Topology topo;
	std::vector<HostBlock> blocks;
};
// Reads deck, topology and every block.  Paths inside the deck and topology are
// resolved relative to `workdir` (the reference resolves them against its CWD).
HostCase load_case(const std::string& deck_path, const std::string& workdir, int n_threads = 0);

}  // namespace e3d
