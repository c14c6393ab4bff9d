// Block sharding of one case over several processes, one GPU each.
//
// The reference distributes blocks over MPI ranks in contiguous ranges
// (BlockCommunicator::BlockCommunicator, MPI/src/BlockCommunicator.cpp:29-38)
// and, once per outer iteration, sends the state of every connexion's origin
// cells to the rank that owns the destination block
// (BlockCommunicator::updateBoundaries, BlockCommunicator.cpp:66-211).
//
// Here a rank's solver holds the blocks of its range.  Connexions with both
// blocks in the range stay device copies (k_halo); the others become halo
// entries that cross the transport: 5 primitives per entry (the reference
// sends 40 variables, of which the ghost cells use only these five).  Both
// sides enumerate the entries the same way, so a send buffer needs no index:
//
//   for each peer rank r (ascending), for each connexion in topology order
//   whose origin block is on the sender and whose destination block is on
//   the receiver, for each cell pair of the connexion in list order
//
// which makes one rank's send segment for r exactly r's receive segment from
// it: the layout of an all-to-all with per-peer counts.
#include <algorithm>

#include "engine.hpp"

namespace e3d {

std::vector<int> shard_first_blocks(int n_blocks, int n_ranks) {
	if (n_ranks < 1) throw Error(E3D_ERR_ARG, "sharding: at least one rank");
	if (n_blocks < n_ranks) throw Error(E3D_ERR_ARG, "sharding: fewer blocks than ranks");
	std::vector<int> first(n_ranks + 1);
	const int n = n_blocks / n_ranks, rem = n_blocks % n_ranks;
	for (int r = 0; r <= n_ranks; r++) first[r] = r * n + std::min(r, rem);
	return first;
}

ShardPlan shard_plan(const HostCase& hc, const std::vector<int>& first_block, int rank) {
	const int nb = (int)hc.blocks.size();
	const int nr = (int)first_block.size() - 1;
	if (nr < 1 || first_block.front() != 0 || first_block.back() != nb)
		throw Error(E3D_ERR_ARG, "sharding: block ranges must start at 0 and end at the block count");
	for (int r = 0; r < nr; r++)
		if (first_block[r + 1] <= first_block[r])
			throw Error(E3D_ERR_ARG, "sharding: every rank needs a non-empty, ascending block range");
	if (rank < 0 || rank >= nr) throw Error(E3D_ERR_ARG, "sharding: rank out of range");
	auto owner = [&](int b) {
		return (int)(std::upper_bound(first_block.begin(), first_block.end(), b) - first_block.begin()) - 1;
	};
	ShardPlan p;
	p.rank = rank;
	p.n_ranks = nr;
	p.first_block = first_block;
	p.b0 = first_block[rank];
	p.b1 = first_block[rank + 1];
	p.send_count.assign(nr, 0);
	p.recv_count.assign(nr, 0);
	for (const Connexion& k : hc.topo.connexions)
		if (owner(k.dest_block) == rank && owner(k.origin_block) == rank) p.local.push_back(k);
	for (int r = 0; r < nr; r++) {
		if (r == rank) continue;
		for (const Connexion& k : hc.topo.connexions) {
			const int od = owner(k.dest_block), oo = owner(k.origin_block);
			if (oo == rank && od == r) {
				for (int c : k.origin_cells) {
					p.send_block.push_back(k.origin_block);
					p.send_cell.push_back(c);
				}
				p.send_count[r] += (long long)k.origin_cells.size();
			}
			if (od == rank && oo == r) {
				for (int c : k.dest_cells) {
					p.recv_block.push_back(k.dest_block);
					p.recv_cell.push_back(c);
				}
				p.recv_count[r] += (long long)k.dest_cells.size();
			}
		}
	}
	return p;
}

}  // namespace e3d
