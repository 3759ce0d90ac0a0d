// Slab plan of the step with the state in host memory (snac_gpu_step_host):
// the slab bounds and the order of the operations on the handle's stream.
// Plain C++ (no CUDA), so that the plan can be checked on the host for
// read-after-write and write-after-read hazards over any mesh and slab count.
//
// The mesh is cut along k (the slowest index of hexes and nodes: hex
// i + j*nx + k*nx*ny, node i + j*(nx+1) + k*(nx+1)*(ny+1)) into S hex slabs
// of whole element blocks and S node slabs of whole node blocks, node slab c
// ending below the first k-plane of hex slab c + 1.  The step is a chain of
// stages alternating between the two kinds of slab (hex, node, hex, ...):
// a hex stage's slab reads the nodes of its k-planes and the next one and
// its own hexes; a node stage's slab reads every hex of its planes and the
// planes below and its own nodes.  Each slab of a stage waits until the
// stage before it has finished what it reads.
#pragma once

#include <algorithm>
#include <vector>

namespace snac {

struct SlabOp {
    enum Kind { KERNEL, UNPACK_REST, NODES_BACK, HEXES_BACK } kind;
    int stage = 0;            // KERNEL: the stage
    int slab = 0;             // KERNEL, HEXES_BACK: the slab
    long long a = 0, b = 0;   // NODES_BACK: node rows [a, b)
};

struct SlabPlan {
    long long ne = 0, nn = 0, LE = 0, P = 0;  // hexes, nodes, hexes per k-layer, nodes per k-plane
    int S = 0, ns = 0;                        // slabs, stages
    std::vector<long long> E, N;              // hex slab c = [E[c], E[c+1]), node slab c = [N[c], N[c+1])
    long long n_head = 0;                     // node rows the first two hex slabs read: uploaded first
    std::vector<SlabOp> ops;                  // in the order they are queued

    // nodes [0, need_nodes(c)) hold every node hex slab c touches
    long long need_nodes(int c) const {
        if (E[c + 1] <= E[c]) return 0;
        const long long k = (E[c + 1] - 1) / LE;
        return std::min(nn, (k + 2) * P);
    }
    // hexes [0, need_elems(d)) hold every hex incident to node slab d
    long long need_elems(int d) const {
        if (N[d + 1] <= N[d]) return 0;
        const long long k = (N[d + 1] - 1) / P;
        return std::min(ne, (k + 1) * LE);
    }
};

// ns stages, even ones over hexes, odd ones over nodes, ns odd (the last is
// the element update, whose slab's hex rows then go back to the host; the
// node rows go back every fourth slab).  Kernels are queued deepest stage
// first, so that a slab's last stage (and its download) is not queued
// behind hex slabs still waiting for their uploads.
inline SlabPlan plan_slabs(long long nx, long long ny, long long nz, int S, int ns, long long hex_block,
                           long long node_block) {
    SlabPlan p;
    p.ne = nx * ny * nz;
    p.nn = (nx + 1) * (ny + 1) * (nz + 1);
    p.LE = nx * ny;
    p.P = (nx + 1) * (ny + 1);
    p.S = S;
    p.ns = ns;
    p.E.assign(S + 1, 0);
    p.N.assign(S + 1, 0);
    for (int c = 0; c < S; c++) {
        p.E[c] = p.ne * c / S / hex_block * hex_block;
        p.N[c] = std::min(p.nn, p.E[c] / p.LE * p.P) / node_block * node_block;
    }
    p.E[S] = p.ne;
    p.N[S] = p.nn;
    p.n_head = std::max(p.need_nodes(0), p.need_nodes(std::min(1, S - 1)));

    std::vector<int> done(ns, 0);
    auto is_node = [](int s) { return (s & 1) != 0; };
    auto ready = [&](int s) -> bool {
        const int i = done[s];
        if (i >= S) return false;
        if (s == 0) return true;
        if (is_node(s)) return p.E[done[s - 1]] >= p.need_elems(i);
        return p.N[done[s - 1]] >= p.need_nodes(i) && done[s - 2] > i;
    };
    bool rest = false;
    long long back = 0;
    for (int total = 0; total < ns * S; total++) {
        int s = ns - 1;
        while (s > 0 && !ready(s)) s--;
        const int i = done[s];
        if (s == 0 && i >= S) break;  // cannot happen: stage 0 always runs to the end
        if (s == 0 && !rest && (i >= 2 || p.need_nodes(i) > p.n_head)) {
            p.ops.push_back({SlabOp::UNPACK_REST});
            rest = true;
        }
        p.ops.push_back({SlabOp::KERNEL, s, i});
        if (s == ns - 1) {
            if ((i + 1) % 4 == 0 || i == S - 1) {
                SlabOp o{SlabOp::NODES_BACK};
                o.a = back;
                o.b = p.N[i + 1];
                p.ops.push_back(o);
                back = p.N[i + 1];
            }
            p.ops.push_back({SlabOp::HEXES_BACK, 0, i});
        }
        done[s]++;
    }
    return p;
}

}  // namespace snac
