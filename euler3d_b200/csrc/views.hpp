// Device-array views shared by the host engine and the kernel translation units.
//
// Cell numbering on the device: all real cells of all blocks first (block after
// block, each in its file order), then all ghost cells (block after block, in
// marker order).  Faces are numbered block after block in the reference's
// creation order.  A "slot" is one (cell, face) incidence; a cell's slots are
// contiguous and follow ascending face id, which is the reference's summation
// order for every per-cell accumulation.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace e3d {

enum GradKind : int { GRAD_GREEN_GAUSS = 0, GRAD_LEAST_SQUARES = 1 };
enum LimKind : int { LIM_BARTH_JESPERSEN = 0, LIM_VENKATAKRISHNAN = 1 };
enum FluxKind : int { FLUX_ROE = 0, FLUX_AUSM = 1 };
enum GhostKind : int { GK_NONE = 0, GK_WALL = 1, GK_FARFIELD = 2, GK_SYMMETRY = 3 };

struct Physics {
	double gamma, gm1, gr;  // gamma, gamma-1, gamma/(gamma-1)
	double cfl;
	double omega, k3;       // BJ shift, Venkatakrishnan K^3
	double free[5];         // freestream rho, u, v, w, p
};

// Mesh topology and FP64 geometry (granular drop-in kernels).
struct GeoView {
	int NR, NG, NA, NF, NS;
	const int* slot_ptr;   // NA+1
	const int* slot_face;  // NS
	const int* slot_nbr;   // NS
	const int* face_lr;    // 2*NF
	const double* S;       // 3*NF area vector, left -> right
	const double* nhat;    // 3*NF S/|S| as the reference normalises it
	const double* area;    // NF
	const double* rl;      // 3*NF
	const double* rr;      // 3*NF
	const double* vol;     // NA
	const double* lsw;     // 3*NS (real-cell slots)
	const signed char* gkind;  // NG boundary-condition kind of each ghost
	const signed char* grefl;  // NG 1: gradient reflected, 0: gradient zero
};

// FP64 state arrays in the reference's meaning (drop-in path).
struct StateView {
	double* prim;  // 5*NA  [var][cell]
	double* rc;    // 5*NR
	double* rd;    // 5*NR
	double* w0;    // 5*NR
	double* grad;  // 15*NA [var][dim][cell]
	double* lim;   // 5*NA
	double* dt;    // NR
	double* srad;  // NR
};

// Fused-path view in working precision T.
template <class T>
struct FusedView {
	int NR, NG, NA, NS;
	int tet4;               // 1 when every real cell has exactly 4 slots (slot = 4c+k)
	const int* slot_ptr;    // NA+1
	const int* slot_nbr;    // NS
	const int* slot_mate;   // NS  >=0: owner is the face's left cell, mate slot index; <0: ~mate, owner is right
	const T* sgeo;          // 4*NS  nx, ny, nz, |S| of the face (face orientation)
	const T* sS;            // 3*NS  area vector signed outward for the owner (Green-Gauss)
	const T* srv;           // 3*NS  r-vector of the owner at the face
	const T* lsw;           // 3*NS  least-squares weights (real slots)
	const T* vol;           // NA
	const signed char* gkind;
	const signed char* grefl;
	const T* Pin;           // 5*NA
	T* Pout;                // 5*NA
	T* FS;                  // 5*NS reconstructed face states [var][slot]
	T* Rc;                  // 5*NR
	T* Rd;                  // 5*NR
	double* W0;             // 5*NR
	T* dt;                  // NR
	const double* case_free;  // 5 per case, or null: every ghost uses Physics::free
	const int* gcase;         // NG case index of each ghost (with case_free)
	// difference form (delta.cu; null otherwise): Pin/Pout hold differences from
	// the base primitives Pb (FP32 copy of Pb64), dW the carried conserved
	// differences from the FP64 base W_b, Rb the FP64-evaluated base residual
	const float* Pb;          // 5*NA
	const double* Pb64;       // 5*NA
	float* dW;                // 5*NR
	float* Rb;                // 5*NR
	const int* slot_face;     // NS  (FP64 face normals of boundary slots)
	const double* nhat64;     // 3*NF
};

// One launch of the persistent batch kernel: several outer iterations over the
// work list (tiles of real cells of the active cases).
struct PersistArgs {
	int n_work;            // work items (tiles)
	const int4* work;      // x: first cell, y: end cell, z: block, w: unused
	const int* block_work; // nblocks+1: work items of block b are [block_work[b], block_work[b+1])
	int nblocks;
	int stages;
	double alpha[5], beta[5];
	int carry;
	int iters;             // outer iterations in this launch
	int start_parity;      // 0: state in P0 (view v0 reads it), 1: state in P1
	int tile_mult;         // a work item covers tile_mult * blockDim cells
	// reductions
	double* wpart;         // n_work*5 per-tile sums of (Rc-Rd)^2
	const int* wall_off;
	const int* wall_face;
	int n_wall;
	double* wall_terms;
	const double* wall_denom;
	double denom;
	const int* face_lr;
	const double* S;
	const double* fc;
	double* hist;          // [iteration][block][10]
	int stride;
	int* d_iter;           // iteration counter (advanced by `iters` at the end)
	int hist_capacity;
	int* d_bad;
	// halo
	int n_halo;
	const int* halo_dst;
	const int* halo_src;
	// difference form: FP64 base primitives (wall pressures are base + difference), else null
	const double* Pb64;
};

}  // namespace e3d
