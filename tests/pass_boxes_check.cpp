// CPU check of the CPML pass boxes (magnelio_b200/csrc/pass_boxes.h) on
// random grids and face layouts: on each side every cell the pass must
// handle is in exactly one box and no other cell is in any; every box's
// face mask equals the slab membership of each of its cells; the block
// ranges match the box sizes.  Layouts: any subset of the six faces in any
// order, slabs from one layer to the whole axis (overlapping low and high
// slabs included), placed as the engine places them (low face at 0, high
// face ending at N).  Exit status 0 when every layout passes.
#include <cstdio>
#include <random>
#include <vector>

#include "pass_boxes.h"

using fitb::PassBoxes;
using fitb::PassFace;

static int check(int nx, int ny, int nz, const std::vector<PassFace>& faces, bool h_side) {
    PassBoxes bx;
    if (!fitb::pass_boxes(bx, nx, ny, nz, faces.data(), (int)faces.size(), h_side)) {
        std::printf("refused: %d x %d x %d, %zu faces\n", nx, ny, nz, faces.size());
        return 1;
    }
    const int top[3] = {nx + 1, ny + 1, nz + 1};
    std::vector<int> cover((size_t)top[0] * top[1] * top[2], 0);
    for (int q = 0; q < bx.n; ++q) {
        long long ncell = 1;
        for (int a = 0; a < 3; ++a) {
            if (bx.lo[q][a] < 0 || bx.hi[q][a] > top[a] || bx.lo[q][a] >= bx.hi[q][a]) {
                std::printf("box %d out of range on axis %d\n", q, a);
                return 1;
            }
            ncell *= bx.hi[q][a] - bx.lo[q][a];
        }
        if (bx.bstart[q + 1] - bx.bstart[q] != (int)((ncell + fitb::kPassThreads - 1) / fitb::kPassThreads)) {
            std::printf("block range of box %d\n", q);
            return 1;
        }
        for (int i = bx.lo[q][0]; i < bx.hi[q][0]; ++i)
            for (int j = bx.lo[q][1]; j < bx.hi[q][1]; ++j)
                for (int k = bx.lo[q][2]; k < bx.hi[q][2]; ++k) {
                    const int c[3] = {i, j, k};
                    unsigned want = 0;
                    for (size_t f = 0; f < faces.size(); ++f) {
                        const int x = c[faces[f].axis];
                        if (x >= faces[f].lo && x < faces[f].lo + faces[f].n) want |= 1u << f;
                    }
                    if (bx.mask[q] != want) {
                        std::printf("mask of box %d at (%d, %d, %d): %x, want %x\n", q, i, j, k, bx.mask[q], want);
                        return 1;
                    }
                    ++cover[((size_t)i * top[1] + j) * top[2] + k];
                }
    }
    for (int i = 0; i < top[0]; ++i)
        for (int j = 0; j < top[1]; ++j)
            for (int k = 0; k < top[2]; ++k) {
                const int c[3] = {i, j, k};
                bool need = false;
                for (const PassFace& f : faces) {
                    const int lo = (h_side && f.lo > 0) ? f.lo - 1 : f.lo;
                    if (c[f.axis] >= lo && c[f.axis] < f.lo + f.n) need = true;
                }
                const int got = cover[((size_t)i * top[1] + j) * top[2] + k];
                if (got != (need ? 1 : 0)) {
                    std::printf("cell (%d, %d, %d) covered %d times, needed %d (%s side)\n", i, j, k, got,
                                need ? 1 : 0, h_side ? "H" : "E");
                    return 1;
                }
            }
    return 0;
}

int main() {
    std::mt19937 rng(2031);
    int layouts = 0;
    for (int trial = 0; trial < 600; ++trial) {
        const int n[3] = {3 + (int)(rng() % 30), 3 + (int)(rng() % 30), 3 + (int)(rng() % 30)};
        std::vector<PassFace> faces;
        for (int side = 0; side < 6; ++side) {
            if (rng() % 3 == 0) continue;  // a random subset of the faces
            const int axis = side / 2, N = n[axis];
            const int thick = 1 + (int)(rng() % N);
            faces.push_back(PassFace{axis, side % 2 == 0 ? 0 : N - thick, thick});
        }
        std::shuffle(faces.begin(), faces.end(), rng);  // face order is the caller's
        for (bool h_side : {false, true}) {
            if (check(n[0], n[1], n[2], faces, h_side)) {
                std::printf("layout %d failed\n", trial);
                return 1;
            }
            ++layouts;
        }
    }
    std::printf("ok %d layouts\n", layouts);
    return 0;
}
