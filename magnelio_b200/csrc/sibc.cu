// Surface-impedance (SIBC) walls on the H update.
//
// Reference: SIBCOperator (src/magnelio/solver/_sibc.py:114-264), called at
// the top of every step (save_field, fit_td.py:837-840) and right after the
// H update and the mu-side ADE, before the H-side CPML corrections
// (update_field, fit_td.py:909-914).  Per face f of a wall with Foster
// branches p:
//   phase 1 (all walls, in wall order):  h_f += beta_H,f (g_f sum_p ((1+k_p)/2) u_p)
//   phase 2 (all walls):                 h_mid = (h_f + h_prev,f) / 2,
//                                        u_p <- k_p u_p;  u_p <- u_p + q_p h_mid
// Phase 2 reads the h that phase 1 completed everywhere (a seam face booked
// by two walls takes both corrections first), so the phases are separate
// launches.  The arithmetic follows the reference's per-array expressions
// in the field dtype, with the branch constants rounded to it.
#include "fitb_common.cuh"

#include <algorithm>

namespace fitb {

namespace {

constexpr int kThreads = 256;

int grid_of(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kThreads - 1) / kThreads, 148LL * 16)); }

template <typename T>
__global__ void k_sibc_save(const T* __restrict__ h, long long blk, int B, SibcDev d) {
    const long long n = d.n_states * B;
    T* hp = static_cast<T*>(d.hprev);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / d.n_states, s = t % d.n_states;
        hp[t] = h[b * blk + d.off[s]];
    }
}

// phase 1: one thread per distinct face; the walls booking it in order
template <typename T>
__global__ void k_sibc_hist(T* __restrict__ h, long long blk, int B, const T* __restrict__ beta, SibcDev d) {
    const long long n = d.n_unique * B;
    const T* g = static_cast<const T*>(d.g);
    const T* u = static_cast<const T*>(d.u);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / d.n_unique, e = t % d.n_unique;
        const long long o = d.uoff[e];
        T v = h[b * blk + o];
        const T be = beta[o];
        for (int r = d.ustart[e]; r < d.ustart[e + 1]; ++r) {
            const long long st = d.ustate[r];
            const int w = d.state_block[st];
            const int p0 = d.br_start[w], p1 = d.br_start[w + 1];
            if (p1 == p0) continue;  // no branches: no history term
            const T* us = u + b * d.n_slots + d.slot[st];
            T hist = (T)d.hopk[p0] * us[0];
            for (int p = p0 + 1; p < p1; ++p) hist = hist + (T)d.hopk[p] * us[p - p0];
            v = v + be * (g[st] * hist);
        }
        h[b * blk + o] = v;
    }
}

// phase 2: one thread per (face, field set)
template <typename T>
__global__ void k_sibc_advance(const T* __restrict__ h, long long blk, int B, SibcDev d) {
    const long long n = d.n_states * B;
    const T* hp = static_cast<const T*>(d.hprev);
    T* u = static_cast<T*>(d.u);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / d.n_states, s = t % d.n_states;
        const int w = d.state_block[s];
        const int p0 = d.br_start[w], p1 = d.br_start[w + 1];
        if (p1 == p0) continue;
        const T hm = T(0.5) * (h[b * blk + d.off[s]] + hp[t]);
        T* us = u + b * d.n_slots + d.slot[s];
        for (int p = p0; p < p1; ++p) {
            T x = us[p - p0] * (T)d.k[p];
            x = x + (T)d.q[p] * hm;
            us[p - p0] = x;
        }
    }
}

}  // namespace

template <typename T>
void launch_sibc_save(const T* h, long long blk, int B, const SibcDev& d, cudaStream_t s) {
    if (d.n_states <= 0) return;
    k_sibc_save<T><<<grid_of(d.n_states * B), kThreads, 0, s>>>(h, blk, B, d);
}

template <typename T>
void launch_sibc_update(T* h, long long blk, int B, const T* beta, const SibcDev& d, cudaStream_t s) {
    if (d.n_states <= 0) return;
    k_sibc_hist<T><<<grid_of(d.n_unique * B), kThreads, 0, s>>>(h, blk, B, beta, d);
    k_sibc_advance<T><<<grid_of(d.n_states * B), kThreads, 0, s>>>(h, blk, B, d);
}

template void launch_sibc_save<float>(const float*, long long, int, const SibcDev&, cudaStream_t);
template void launch_sibc_save<double>(const double*, long long, int, const SibcDev&, cudaStream_t);
template void launch_sibc_update<float>(float*, long long, int, const float*, const SibcDev&, cudaStream_t);
template void launch_sibc_update<double>(double*, long long, int, const double*, const SibcDev&, cudaStream_t);

}  // namespace fitb
