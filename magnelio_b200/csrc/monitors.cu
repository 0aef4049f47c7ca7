// Running-DFT field monitors, blocked in time.
//
// Reference: MonitorFieldFrequency.record
// (src/magnelio/monitors/field_frequency.py:249-294) interpolates the
// staggered states to cell centres (src/magnelio/monitors/base.py:51-168)
// and adds bins[f] += exp(j w_f t) dt_w * data (src/magnelio/monitors/_dft.py
// :37-52) every recorded step, with t = n dt for E and (n + 1/2) dt for H.
//
// Here each recorded step only stages the interpolated float32 samples and
// the float64-evaluated phasors exp(j w t) dt_w of that step into a block of
// K slots (k_dft_stage_all).  When a monitor's block is full,
// k_dft_flush_all forms sum_s w_s[f] x_s for every bin in registers and adds
// it once to the bins (optionally Kahan-compensated): the complex bins are
// read and written once per K recorded steps instead of once per step.
// All monitors share one stage launch and one flush launch per step; the
// last CTA of the flush launch advances the device step counter.
#include "fitb_common.cuh"

namespace fitb {

namespace {

constexpr int kMaxK = 32;
constexpr int kThreads = 256;

__device__ __forceinline__ long long recorded_upto(long long x, int stride) {
    // Number of steps n' in [0, x] with n' % stride == 0 (0 for x < 0).
    return (x < 0) ? 0 : x / stride + 1;
}

template <typename T>
__device__ __forceinline__ double interp_sample(const T* E, const T* H, long long vol, const Geom& g,
                                                const DftDev& d, int c, int i, int j, int k) {
    const long long o = pidx(g, i, j, k);
    const double* dx = d.inv;
    const double* dy = d.inv + d.inv_ld;
    const double* dz = d.inv + 2 * d.inv_ld;
    const double* dxa = d.dual;
    const double* dya = d.dual + d.inv_ld;
    const double* dza = d.dual + 2 * d.inv_ld;
    const long long si = g.si, sj = g.sj;
    switch (c) {
        case 0: {
            const T* A = E;
            T s = ((A[o] + A[o + sj]) + A[o + 1]) + A[o + sj + 1];
            return (double)(T(0.25) * s) / dx[i];
        }
        case 1: {
            const T* A = E + vol;
            T s = ((A[o] + A[o + si]) + A[o + 1]) + A[o + si + 1];
            return (double)(T(0.25) * s) / dy[j];
        }
        case 2: {
            const T* A = E + 2 * vol;
            T s = ((A[o] + A[o + si]) + A[o + sj]) + A[o + si + sj];
            return (double)(T(0.25) * s) / dz[k];
        }
        case 3: {
            const T* A = H;
            return 0.5 * ((double)A[o] / dxa[i] + (double)A[o + si] / dxa[i + 1]);
        }
        case 4: {
            const T* A = H + vol;
            return 0.5 * ((double)A[o] / dya[j] + (double)A[o + sj] / dya[j + 1]);
        }
        default: {
            const T* A = H + 2 * vol;
            return 0.5 * ((double)A[o] / dza[k] + (double)A[o + 1] / dza[k + 1]);
        }
    }
}

__device__ __forceinline__ int monitor_of_block(const DftDev* devs, int nmon, bool stage) {
    int m = 0;
    while (m + 1 < nmon && (int)blockIdx.x >= (stage ? devs[m + 1].sblk0 : devs[m + 1].fblk0)) ++m;
    return m;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
    k_dft_stage_all(const T* __restrict__ e, const T* __restrict__ h, long long e_block, long long h_block, Geom g,
                    int B, const DftDev* __restrict__ devs, int nmon, const long long* __restrict__ step) {
    const DftDev& d = devs[monitor_of_block(devs, nmon, true)];
    const int lb = blockIdx.x - d.sblk0;
    const long long n = *step;
    if (n % d.stride) return;
    const long long cnt = recorded_upto(n, d.stride) - recorded_upto(*d.base - 1, d.stride);
    const int slot = (int)((cnt - 1) % d.K);
    if (lb == 0) {
        const double tE = (double)n * d.dt;
        const double tH = tE + 0.5 * d.dt;
        const double dtw = (double)d.stride * d.dt;
        for (int q = threadIdx.x; q < 2 * d.nf; q += blockDim.x) {
            const int f = q % d.nf;
            const double t = (q < d.nf) ? tE : tH;
            double sn, cs;
            sincos(d.omega[f] * t, &sn, &cs);
            d.wst[((long long)slot * 2 + (q / d.nf)) * d.nf + f] = make_float2((float)(cs * dtw), (float)(sn * dtw));
        }
    }
    const long long total = (long long)d.ncomp * d.ncell;
    for (long long t = lb * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)d.sblk * blockDim.x) {
        const int ci = (int)(t / d.ncell);
        const long long cell = t % d.ncell;
        const int kk = (int)(cell % d.nk);
        const long long r = cell / d.nk;
        const int jj = (int)(r % d.nj);
        const int ii = (int)(r / d.nj);
        const int c = d.comps[ci];
        for (int b = 0; b < B; ++b) {
            const double v = interp_sample<T>(e + (long long)b * e_block, h + (long long)b * h_block, g.vol, g, d, c,
                                              d.i0 + ii, d.j0 + jj, d.k0 + kk);
            d.stage[(((long long)b * d.K + slot) * d.ncomp + ci) * d.ncell + cell] = (float)v;
        }
    }
}

// Adds the kc staged slots of one monitor to its bins (threads of the
// monitor's blocks, lb = local block index, nb = the monitor's block count).
__device__ void flush_slots(int B, const DftDev& d, int kc, int lb, int nb, float2* sw) {
    for (int q = threadIdx.x; q < kc * 2 * d.nf; q += blockDim.x) sw[q] = d.wst[q];
    __syncthreads();
    const long long per_b = (long long)d.ncomp * d.ncell;
    const long long total = (long long)B * per_b;
    for (long long t = lb * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)nb * blockDim.x) {
        const int b = (int)(t / per_b);
        const long long r = t % per_b;
        const int ci = (int)(r / d.ncell);
        const long long cell = r % d.ncell;
        const int tsel = (d.comps[ci] < 3) ? 0 : 1;
        float x[kMaxK];
#pragma unroll
        for (int s = 0; s < kMaxK; ++s)
            x[s] = (s < kc) ? d.stage[(((long long)b * d.K + s) * d.ncomp + ci) * d.ncell + cell] : 0.0f;
        for (int f = 0; f < d.nf; ++f) {
            float re = 0.0f, im = 0.0f;
#pragma unroll
            for (int s = 0; s < kMaxK; ++s) {
                if (s < kc) {
                    const float2 w = sw[(s * 2 + tsel) * d.nf + f];
                    re = fmaf(w.x, x[s], re);
                    im = fmaf(w.y, x[s], im);
                }
            }
            const long long bi = (((long long)b * d.ncomp + ci) * d.nf + f) * d.ncell + cell;
            float2 acc = d.bins[bi];
            if (d.kahan) {
                float2 cm = d.cmp[bi];
                const float yr = re - cm.x, yi = im - cm.y;
                const float tr = acc.x + yr, ti = acc.y + yi;
                cm.x = (tr - acc.x) - yr;
                cm.y = (ti - acc.y) - yi;
                acc.x = tr;
                acc.y = ti;
                d.cmp[bi] = cm;
            } else {
                acc.x += re;
                acc.y += im;
            }
            d.bins[bi] = acc;
        }
    }
}

__global__ void __launch_bounds__(kThreads)
    k_dft_flush_all(int B, const DftDev* __restrict__ devs, int nmon, long long* step, unsigned* ticket) {
    extern __shared__ float2 sw[];
    const DftDev& d = devs[monitor_of_block(devs, nmon, false)];
    const int lb = blockIdx.x - d.fblk0;
    const long long n = *step;
    bool go = (n % d.stride) == 0;
    if (go) {
        const long long cnt = recorded_upto(n, d.stride) - recorded_upto(*d.base - 1, d.stride);
        go = (int)((cnt - 1) % d.K) == d.K - 1;
    }
    if (go) flush_slots(B, d, d.K, lb, d.fblk, sw);
    // The last CTA to finish advances the step counter: every CTA has read
    // it above, and the next launch in the stream starts after this one.
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(ticket, 1u) == gridDim.x - 1) {
            *ticket = 0u;
            step[0] = n + 1;
            __threadfence();
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_dft_flush_forced(int B, DftDev d, int kc) {
    extern __shared__ float2 sw[];
    flush_slots(B, d, kc, blockIdx.x, gridDim.x, sw);
}

}  // namespace

int dft_blocks(long long work) {
    long long b = (work + kThreads - 1) / kThreads;
    if (b > 148 * 4) b = 148 * 4;
    return (int)(b < 1 ? 1 : b);
}

template <typename T>
void launch_dft_stage_all(const T* e, const T* h, long long e_block, long long h_block, const Geom& g, int B,
                          const DftDev* devs, int nmon, int nblocks, const long long* step, cudaStream_t s) {
    k_dft_stage_all<T><<<nblocks, kThreads, 0, s>>>(e, h, e_block, h_block, g, B, devs, nmon, step);
}

void launch_dft_flush_all(int B, const DftDev* devs, int nmon, int nblocks, size_t smem, long long* step,
                          unsigned* ticket, cudaStream_t s) {
    k_dft_flush_all<<<nblocks, kThreads, smem, s>>>(B, devs, nmon, step, ticket);
}

void launch_dft_flush_forced(int B, const DftDev& d, int kc, cudaStream_t s) {
    const size_t smem = (size_t)kc * 2 * d.nf * sizeof(float2);
    k_dft_flush_forced<<<dft_blocks((long long)B * d.ncomp * d.ncell), kThreads, smem, s>>>(B, d, kc);
}

template void launch_dft_stage_all<float>(const float*, const float*, long long, long long, const Geom&, int,
                                          const DftDev*, int, int, const long long*, cudaStream_t);
template void launch_dft_stage_all<double>(const double*, const double*, long long, long long, const Geom&, int,
                                           const DftDev*, int, int, const long long*, cudaStream_t);

}  // namespace fitb
