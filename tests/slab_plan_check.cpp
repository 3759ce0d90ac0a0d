// Host-side check of the slab plan of snac_gpu_step_host
// (snac_b200/csrc/snac_slab_plan.h): every operation, in the plan's order,
// reads node and hex rows at exactly the version the whole-mesh step would
// give it (no read-after-write or write-after-read hazard), reads only rows
// already uploaded, and every row goes back to the host once, final.
//
// Versions: -1 = as uploaded; s = written by stage s.  A hex stage s reads
// the nodes of its hexes at the version of node stage s-1 and its own hexes
// at the version of hex stage s-2; a node stage s reads the hexes incident
// to its nodes at the version of hex stage s-1 and its own nodes at the
// version of node stage s-2.
//
// Usage: slab_plan_check  -> prints "ok <cases>" and exits 0, or the first
// failing case and exits 1.
#include <cstdio>
#include <vector>

#include "snac_slab_plan.h"

using snac::SlabOp;
using snac::SlabPlan;

static int check(long long nx, long long ny, long long nz, int S, int ns) {
    const SlabPlan p = snac::plan_slabs(nx, ny, nz, S, ns, 12, 128);
    const long long ne = p.ne, nn = p.nn, nnx = nx + 1, nny = ny + 1;
    std::vector<int> nv(nn, -1), hv(ne, -1);
    std::vector<char> hex_up(ne, 0), node_back(nn, 0), hex_back(ne, 0);
    long long node_up = p.n_head;  // node rows [0, node_up) are on the device
    std::vector<int> done(ns, 0);
    auto fail = [&](const char* what, long long idx) {
        std::printf("FAIL %s at %lld: mesh %lldx%lldx%lld, %d slabs, %d stages\n", what, idx, nx, ny, nz, S, ns);
        return 1;
    };
    auto corner = [&](long long e, int c) {
        const long long i = e % nx, j = (e / nx) % ny, k = e / (nx * ny);
        return (i + (c & 1)) + (j + ((c >> 1) & 1)) * nnx + (k + ((c >> 2) & 1)) * nnx * nny;
    };
    for (const SlabOp& o : p.ops) {
        if (o.kind == SlabOp::UNPACK_REST) {
            node_up = nn;
            continue;
        }
        if (o.kind == SlabOp::NODES_BACK) {
            for (long long n = o.a; n < o.b; n++) {
                if (nv[n] != ns - 2) return fail("node row sent back before its last stage", n);
                if (node_back[n]++) return fail("node row sent back twice", n);
            }
            continue;
        }
        if (o.kind == SlabOp::HEXES_BACK) {
            for (long long e = p.E[o.slab]; e < p.E[o.slab + 1]; e++) {
                if (hv[e] != ns - 1) return fail("hex row sent back before its last stage", e);
                if (hex_back[e]++) return fail("hex row sent back twice", e);
            }
            continue;
        }
        const int s = o.stage, i = o.slab;
        if (i != done[s]++) return fail("slabs of a stage out of order", i);
        if ((s & 1) == 0) {  // hex stage
            if (s == 0)
                for (long long e = p.E[i]; e < p.E[i + 1]; e++) hex_up[e] = 1;  // the slab's upload event
            for (long long e = p.E[i]; e < p.E[i + 1]; e++) {
                if (!hex_up[e]) return fail("hex read before its upload", e);
                if (hv[e] != (s >= 2 ? s - 2 : -1)) return fail("hex read at the wrong version", e);
                for (int c = 0; c < 8; c++) {
                    const long long n = corner(e, c);
                    if (n >= node_up) return fail("node read before its upload", n);
                    if (nv[n] != s - 1) return fail("node read at the wrong version", n);
                }
            }
            for (long long e = p.E[i]; e < p.E[i + 1]; e++) hv[e] = s;
        } else {  // node stage
            for (long long n = p.N[i]; n < p.N[i + 1]; n++) {
                if (n >= node_up) return fail("node read before its upload", n);
                if (nv[n] != (s >= 2 ? s - 2 : -1)) return fail("own node read at the wrong version", n);
                const long long ii = n % nnx, jj = (n / nnx) % nny, kk = n / (nnx * nny);
                for (int c = 0; c < 8; c++) {
                    const long long ei = ii - 1 + (c & 1), ej = jj - 1 + ((c >> 1) & 1), ek = kk - 1 + ((c >> 2) & 1);
                    if (ei < 0 || ej < 0 || ek < 0 || ei >= nx || ej >= ny || ek >= nz) continue;
                    const long long e = ei + ej * nx + ek * nx * ny;
                    if (hv[e] != s - 1) return fail("incident hex read at the wrong version", e);
                }
            }
            for (long long n = p.N[i]; n < p.N[i + 1]; n++) nv[n] = s;
        }
    }
    for (int s = 0; s < ns; s++)
        if (done[s] != S) return fail("stage left unfinished", s);
    for (long long n = 0; n < nn; n++)
        if (!node_back[n]) return fail("node row never sent back", n);
    for (long long e = 0; e < ne; e++)
        if (!hex_back[e]) return fail("hex row never sent back", e);
    return 0;
}

int main() {
    const long long meshes[][3] = {{1, 1, 1},  {1, 3, 1},  {2, 1, 5},  {3, 2, 1},   {7, 1, 1},  {1, 1, 40},
                                   {5, 3, 7},  {13, 5, 11}, {8, 4, 8},  {6, 4, 6},   {3, 3, 100}, {16, 8, 16},
                                   {17, 9, 23}, {64, 32, 64}};
    int cases = 0;
    for (const auto& mesh : meshes)
        for (int ns : {3, 5})
            for (int S = 1; S <= 64; S += (S < 20 ? 1 : 11)) {
                if (check(mesh[0], mesh[1], mesh[2], S, ns)) return 1;
                cases++;
            }
    std::printf("ok %d\n", cases);
    return 0;
}
