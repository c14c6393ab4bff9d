// Order-preserving hash replacement for the reference's quadratic face search.
//
// Test infrastructure (oracle build only).  The reference builds faces in
// ConcreteBlockBuilder::createMyFaces (BlockBuilder/src/ConcreteBlockBuilder.cpp:497-742)
// by visiting real cells in ascending id, asking each cell's local face table
// (FactoryMethod/src/Temp*FaceCreator.cpp) for its faces in table order, and
// comparing every candidate against every face already built (O(F^2)); a face
// is created on its first occurrence and keeps the node order of that
// occurrence.  Two faces match when they have the same node count and the same
// node set (the 6 / 24 permutation tables at :522-534).
//
// This definition keeps exactly that visiting order, the first-occurrence rule,
// the node order and the face ids, and replaces only the search by a hash of the
// sorted node ids.  It is linked with a strong symbol over the weakened original,
// so every other reference object is used unchanged.
#include "ConcreteBlockBuilder.h"
#include "TempTetrahedralFaceCreator.h"
#include "TempPrismFaceCreator.h"
#include "TempPyramidFaceCreator.h"
#include "TempFaceCreator.h"
#include "FaceCreator.h"
#include "Block.h"
#include "Cell.h"
#include "Face.h"

#include <algorithm>
#include <array>
#include <cstdint>
#include <iostream>
#include <unordered_set>

namespace {

struct FaceKey {
	std::array<int, 4> n;  // sorted node ids, -1 padded for triangles
	bool operator==(const FaceKey& o) const { return n == o.n; }
};

struct FaceKeyHash {
	size_t operator()(const FaceKey& k) const {
		uint64_t h = 1469598103934665603ull;
		for (int v : k.n) {
			h ^= static_cast<uint64_t>(static_cast<uint32_t>(v));
			h *= 1099511628211ull;
		}
		return static_cast<size_t>(h);
	}
};

}  // namespace

void ConcreteBlockBuilder::createMyFaces(Block* block)
{
	TempTetrahedralFaceCreator tetrahedral_face_creator = TempTetrahedralFaceCreator();
	TempPrismFaceCreator prism_face_creator = TempPrismFaceCreator();
	TempPyramidFaceCreator pyramid_face_creator = TempPyramidFaceCreator();
	// same creator-key indexing as the reference (0 tet, 1 pyramid, 2 hexahedron)
	TempFaceCreator temp_face_creators[3];
	temp_face_creators[0] = tetrahedral_face_creator;
	temp_face_creators[1] = pyramid_face_creator;
	temp_face_creators[2] = prism_face_creator;
	FaceCreator* real_face_creator = new FaceCreator();

	std::unordered_set<FaceKey, FaceKeyHash> seen;
	seen.reserve(static_cast<size_t>(block->n_faces_in_block_) * 2 + 16);

	for (int i = 0; i < block->n_real_cells_in_block_; i++) {
		Cell* cell = block->block_cells_[i];
		Face** temp_faces = temp_face_creators[cell->creator_key_].createFace(cell);
		for (int j = 0; j < cell->n_faces_per_cell_; j++) {
			Face* face = temp_faces[j];
			const int nn = face->n_nodes_per_face_;
			FaceKey key;
			key.n = {-1, -1, -1, -1};
			for (int k = 0; k < nn && k < 4; k++) key.n[k] = face->face_2_nodes_connectivity_[k];
			std::sort(key.n.begin(), key.n.begin() + std::min(nn, 4));
			if (seen.insert(key).second) {
				Face* new_face = buildFace(face_count_, nn, real_face_creator);
				new_face->block_id_ = block->block_id_;
				for (int k = 0; k < nn; k++)
					new_face->face_2_nodes_connectivity_[k] = face->face_2_nodes_connectivity_[k];
				block->addFace(new_face);
				face_count_ += 1;
			}
			delete face;
		}
		delete[] temp_faces;
	}
	if (face_count_ != block->n_faces_in_block_) {
		std::cerr << "fast_faces: built " << face_count_ << " faces, pre-read counted "
		          << block->n_faces_in_block_ << std::endl;
	}
	delete real_face_creator;
}
