// ADE pole-current update for dispersive materials (reference:
// solver/_dispersion.py:504-569, called from fit_td.py:833-859, :906-907),
// and the CPML correction as a separate pass for the sides that have one.
//
// Per side (E: eps(omega) on E edges, H: mu(omega) on H faces):
//   save      f_prev[s] = f[off[s]]                      (top of the step)
//   subtract  f[o] -= beta[o] * sum_p (w_p/2) Re((1 + k_p) J_p[s])
//             for every state s on entry o, in block order (entries that
//             two materials share take both blocks' terms in turn)
//   advance   J_p[s] = J_p[s] k_p + c_p g[s] (f[off[s]] - f_prev[s])
// States and g are stored in the field dtype, k_p / c_p in float64, and the
// recursions run in float64 with every product and sum rounded as written
// (no contraction), as the reference's fused CPU kernels do (single
// storage, double operations).
//
// The reference applies the CPML corrections after this update
// (fit_td.py:858-874): on a side with dispersion the stencil kernel runs
// without its fused CPML and k_cpml_pass applies it face by face here.
#include "fitb_common.cuh"

namespace fitb {

namespace {

template <typename T>
__global__ void k_disp_save(const T* __restrict__ F, long long blk, int B, const DispDev d) {
    const long long work = (long long)d.n_states * B;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < work;
         q += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(q / d.n_states);
        const long long s = q - (long long)b * d.n_states;
        static_cast<T*>(d.fprev)[q] = F[b * blk + d.off[s]];
    }
}

// history current of state s (sum over its block's poles, pole order)
template <typename T>
__device__ __forceinline__ double j_hist(const DispDev& d, int b, long long s) {
    const int blk = d.state_block[s];
    const int q0 = d.pole_start[blk], q1 = d.pole_start[blk + 1];
    const T* J = static_cast<const T*>(d.J) + (long long)b * d.n_slots + d.slot[s];
    double jh = 0.0;
    for (int q = q0; q < q1; ++q) {
        const T* js = J + 2 * (q - q0);
        double term;
        if (d.kind[q] == 0) {
            term = __dmul_rn(d.hw[q], __dmul_rn(d.opk_re[q], (double)js[0]));
        } else {
            const double re = __dsub_rn(__dmul_rn(d.opk_re[q], (double)js[0]), __dmul_rn(d.opk_im[q], (double)js[1]));
            term = __dmul_rn(d.hw[q], re);
        }
        jh = q == q0 ? term : __dadd_rn(jh, term);
    }
    return jh;
}

template <typename T>
__global__ void k_disp_subtract(T* F, long long blk, int B, const T* __restrict__ beta, const DispDev d) {
    const long long work = (long long)d.n_unique * B;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < work;
         q += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(q / d.n_unique);
        const long long u = q - (long long)b * d.n_unique;
        const long long o = d.uoff[u];
        T v = F[b * blk + o];
        const double bt = (double)beta[o];
        for (int r = d.ustart[u]; r < d.ustart[u + 1]; ++r) {
            const double jh = j_hist<T>(d, b, d.ustate[r]);
            v = (T)__dsub_rn((double)v, __dmul_rn(bt, jh));
        }
        F[b * blk + o] = v;
    }
}

template <typename T>
__device__ __forceinline__ T sub_rn(T a, T b);
template <>
__device__ __forceinline__ float sub_rn<float>(float a, float b) { return __fsub_rn(a, b); }
template <>
__device__ __forceinline__ double sub_rn<double>(double a, double b) { return __dsub_rn(a, b); }
template <typename T>
__device__ __forceinline__ T mul_rn(T a, T b);
template <>
__device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <>
__device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }

template <typename T>
__global__ void k_disp_advance(const T* __restrict__ F, long long blk, int B, const DispDev d) {
    const long long work = (long long)d.n_states * B;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < work;
         q += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(q / d.n_states);
        const long long s = q - (long long)b * d.n_states;
        const T fp = static_cast<const T*>(d.fprev)[q];
        const T gd = mul_rn<T>(static_cast<const T*>(d.g)[s], sub_rn<T>(F[b * blk + d.off[s]], fp));
        const double g64 = (double)gd;
        const int bk = d.state_block[s];
        const int q0 = d.pole_start[bk], q1 = d.pole_start[bk + 1];
        T* J = static_cast<T*>(d.J) + (long long)b * d.n_slots + d.slot[s];
        for (int p = q0; p < q1; ++p) {
            T* js = J + 2 * (p - q0);
            if (d.kind[p] == 0) {
                js[0] = (T)__dadd_rn(__dmul_rn((double)js[0], d.k_re[p]), __dmul_rn(d.c_re[p], g64));
            } else {
                const double jr = (double)js[0], ji = (double)js[1];
                const double mr = __dsub_rn(__dmul_rn(jr, d.k_re[p]), __dmul_rn(ji, d.k_im[p]));
                const double mi = __dadd_rn(__dmul_rn(jr, d.k_im[p]), __dmul_rn(ji, d.k_re[p]));
                js[0] = (T)__dadd_rn(mr, __dmul_rn(d.c_re[p], g64));
                js[1] = (T)__dadd_rn(mi, __dmul_rn(d.c_im[p], g64));
            }
        }
    }
}

// One CPML face, one side, as a pass over its slab (cpml.py:343-516): the
// same psi recursion and correction as the fused form in the stencil
// kernels, applied after the side's other updates.
template <typename T>
__global__ void k_cpml_pass(const StencilArgs<T> a, int q, int side) {
    const Geom& g = a.g;
    const FaceDev& f = a.f[q];
    const long long vol = g.vol, fs = 3 * vol;
    const long long work = f.slab * a.B;
    const T* bcc = static_cast<const T*>(f.bcc);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < work;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / f.slab);
        const long long s = t - (long long)b * f.slab;
        const int c = (int)(s % f.pk);
        if (c >= f.dK) continue;  // row pitch padding
        const long long r = s / f.pk;
        const int bb = (int)(r % f.dJ), aa = (int)(r / f.dJ);
        const int l = f.axis == 0 ? aa : (f.axis == 1 ? bb : c);
        const int i = f.axis == 0 ? f.lo + aa : aa;
        const int j = f.axis == 1 ? f.lo + bb : bb;
        const int k = f.axis == 2 ? f.lo + c : c;
        const long long o = pidx(g, i, j, k);
        const long long sa = f.axis == 0 ? g.si : (f.axis == 1 ? g.sj : 1);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        T* psi = static_cast<T*>(f.psi) + (long long)b * 4 * f.slab;
        if (side == 0) {
            const T* H = a.h + b * fs;
            T* E = a.e + b * fs;
            // transverse H components of this axis: (first, second)
            const long long c1 = f.axis == 2 ? vol : 2 * vol;      // Hz, Hz, Hy
            const long long c2 = f.axis == 0 ? vol : 0;            // Hy, Hx, Hx
            const T d1 = H[c1 + o] - H[c1 + o - sa];
            const T d2 = H[c2 + o] - H[c2 + o - sa];
            T p1 = psi[s] * cb;
            p1 = p1 + cc * d1;
            if (!f.air[s]) p1 = T(0);
            psi[s] = p1;
            T p2 = psi[f.slab + s] * cb;
            p2 = p2 + cc * d2;
            if (!f.air[f.slab + s]) p2 = T(0);
            psi[f.slab + s] = p2;
            const T bx = a.bE[o], by = a.bE[vol + o], bz = a.bE[2 * vol + o];
            if (f.axis == 0) {
                E[vol + o] = E[vol + o] + by * (cck * d1 + p1);
                E[2 * vol + o] = E[2 * vol + o] - bz * (cck * d2 + p2);
            } else if (f.axis == 1) {
                E[o] = E[o] - bx * (cck * d1 + p1);
                E[2 * vol + o] = E[2 * vol + o] + bz * (cck * d2 + p2);
            } else {
                E[o] = E[o] + bx * (cck * d1 + p1);
                E[vol + o] = E[vol + o] - by * (cck * d2 + p2);
            }
        } else {
            const T* E = a.e + b * fs;
            T* H = a.h + b * fs;
            const long long c1 = f.axis == 2 ? vol : 2 * vol;      // Ez, Ez, Ey
            const long long c2 = f.axis == 0 ? vol : 0;            // Ey, Ex, Ex
            const T d1 = E[c1 + o + sa] - E[c1 + o];
            const T d2 = E[c2 + o + sa] - E[c2 + o];
            const long long s1 = 2 * f.slab + s, s2 = 3 * f.slab + s;
            T p1 = psi[s1] * cb;
            p1 = p1 + cc * d1;
            if (!f.air[s1]) p1 = T(0);
            psi[s1] = p1;
            T p2 = psi[s2] * cb;
            p2 = p2 + cc * d2;
            if (!f.air[s2]) p2 = T(0);
            psi[s2] = p2;
            const T bx = a.bH[o], by = a.bH[vol + o], bz = a.bH[2 * vol + o];
            if (f.axis == 0) {
                H[vol + o] = H[vol + o] - by * (cck * d1 + p1);
                H[2 * vol + o] = H[2 * vol + o] + bz * (cck * d2 + p2);
            } else if (f.axis == 1) {
                H[o] = H[o] + bx * (cck * d1 + p1);
                H[2 * vol + o] = H[2 * vol + o] - bz * (cck * d2 + p2);
            } else {
                H[o] = H[o] - bx * (cck * d1 + p1);
                H[vol + o] = H[vol + o] + by * (cck * d2 + p2);
            }
        }
    }
}

int grid_for(long long work) {
    const long long want = (work + 255) / 256;
    return (int)(want < 148 * 8 ? (want < 1 ? 1 : want) : 148 * 8);
}

}  // namespace

template <typename T>
void launch_disp_save(const T* F, long long blk, int B, const DispDev& d, cudaStream_t s) {
    if (d.n_states <= 0) return;
    k_disp_save<T><<<grid_for(d.n_states * B), 256, 0, s>>>(F, blk, B, d);
}
template <typename T>
void launch_disp_update(T* F, long long blk, int B, const T* beta, const DispDev& d, cudaStream_t s) {
    if (d.n_states <= 0) return;
    k_disp_subtract<T><<<grid_for(d.n_unique * B), 256, 0, s>>>(F, blk, B, beta, d);
    k_disp_advance<T><<<grid_for(d.n_states * B), 256, 0, s>>>(F, blk, B, d);
}
template <typename T>
void launch_cpml_pass(const StencilArgs<T>& a, int q, int side, cudaStream_t s) {
    k_cpml_pass<T><<<grid_for(a.f[q].slab * a.B), 256, 0, s>>>(a, q, side);
}
template void launch_disp_save<float>(const float*, long long, int, const DispDev&, cudaStream_t);
template void launch_disp_save<double>(const double*, long long, int, const DispDev&, cudaStream_t);
template void launch_disp_update<float>(float*, long long, int, const float*, const DispDev&, cudaStream_t);
template void launch_disp_update<double>(double*, long long, int, const double*, const DispDev&, cudaStream_t);
template void launch_cpml_pass<float>(const StencilArgs<float>&, int, int, cudaStream_t);
template void launch_cpml_pass<double>(const StencilArgs<double>&, int, int, cudaStream_t);

}  // namespace fitb
