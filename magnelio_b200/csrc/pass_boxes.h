// Disjoint cell boxes of the CPML slab passes of the tile step
// (stencil_tile.cu).  Host-only code, shared with the CPU check of its
// invariants (tests/pass_boxes_check.cpp).
#pragma once

#include <algorithm>
#include <vector>

namespace fitb {

// Disjoint cell boxes [lo, hi) of a CPML pass, each with the CPML faces
// (bit q = face q) of all its cells.  Blocks of 256 threads cover 256
// consecutive cells of one box (k fastest): block ranges bstart.
constexpr int kPassThreads = 256;
constexpr int kMaxPassBoxes = 128;  // six faces: at most 4^3 - 8 (E side), 5^3 - 8 (H side)
struct PassBoxes {
    int n;
    int lo[kMaxPassBoxes][3], hi[kMaxPassBoxes][3];
    unsigned mask[kMaxPassBoxes];
    int bstart[kMaxPassBoxes + 1];
};

// A CPML face: its axis (0 = x, 1 = y, 2 = z) and its slab [lo, lo + n).
struct PassFace {
    int axis, lo, n;
};

// Disjoint boxes of the CPML passes.  Along each axis the cells split into
// segments by the faces of that axis: the slab of each face (E side), or
// the slab with one more layer on its low side (H side: the H cells whose
// curl takes a slab E edge at i+1, j+1 or k+1, recomputed with the E the
// CPML corrected); a segment carries the faces whose actual slab contains
// it.  The boxes are the products of segments that some face reaches.
// Returns false when there are more boxes than the table holds.
inline bool pass_boxes(PassBoxes& bx, int nx, int ny, int nz, const PassFace* f, int nfaces, bool h_side) {
    bx = PassBoxes{};
    const int top[3] = {nx + 1, ny + 1, nz + 1};
    struct Seg {
        int lo, hi;
        unsigned faces;  // actual slab membership
        bool reach;      // inside some (extended) range of this axis
    };
    std::vector<Seg> segs[3];
    for (int a = 0; a < 3; ++a) {
        std::vector<int> cuts = {0, top[a]};
        for (int q = 0; q < nfaces; ++q) {
            if (f[q].axis != a) continue;
            const int lo = f[q].lo, hi = std::min(f[q].lo + f[q].n, top[a]);
            cuts.push_back(lo);
            cuts.push_back(hi);
            if (h_side && lo > 0) cuts.push_back(lo - 1);
        }
        std::sort(cuts.begin(), cuts.end());
        cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
        for (size_t c = 0; c + 1 < cuts.size(); ++c) {
            Seg sg{cuts[c], cuts[c + 1], 0u, false};
            for (int q = 0; q < nfaces; ++q) {
                if (f[q].axis != a) continue;
                const int lo = f[q].lo, hi = std::min(f[q].lo + f[q].n, top[a]);
                if (sg.lo >= lo && sg.hi <= hi) sg.faces |= 1u << q;  // overlapping slabs: both, face order
                const int elo = (h_side && lo > 0) ? lo - 1 : lo;
                if (sg.lo >= elo && sg.hi <= hi) sg.reach = true;
            }
            segs[a].push_back(sg);
        }
    }
    int acc = 0;
    for (const Seg& x : segs[0])
        for (const Seg& y : segs[1])
            for (const Seg& z : segs[2]) {
                if (!(x.reach || y.reach || z.reach)) continue;
                if (bx.n == kMaxPassBoxes) return false;
                const int q = bx.n++;
                bx.lo[q][0] = x.lo;
                bx.hi[q][0] = x.hi;
                bx.lo[q][1] = y.lo;
                bx.hi[q][1] = y.hi;
                bx.lo[q][2] = z.lo;
                bx.hi[q][2] = z.hi;
                bx.mask[q] = x.faces | y.faces | z.faces;
                const long long ncell = (long long)(x.hi - x.lo) * (y.hi - y.lo) * (z.hi - z.lo);
                if (ncell >= (1LL << 31)) return false;
                bx.bstart[q] = acc;
                acc += (int)((ncell + kPassThreads - 1) / kPassThreads);
            }
    bx.bstart[bx.n] = acc;
    return true;
}

}  // namespace fitb
