// Modal S-parameters from the device-resident port records, on the device.
//
// Reference: compute_s_parameters (src/magnelio/post/modal_sparameters.py
// :335-545) over Signal1D.at_frequencies (src/magnelio/signals/
// signal_1d.py:59-97, the direct DFT sum_n x_n exp(-2 pi j f n dt)), the Yee
// half-step alignment of I (exp(+j omega dt / 2) unless the channel samples
// I with V), the per-channel power-wave split and S = b / a_excited with the
// bins where |a_excited| falls below a_threshold of its peak set to NaN.
// The power-wave split is linear in (V(f), I(f)) with per-channel,
// per-frequency coefficients that come from the port's mode; the caller
// passes them (maps[c] = aV, aI, bV, bI), as magnelio_b200/sparams.py does
// on the host.
//
// Stage 1 (k_vi_dft): one CTA per (block of kFB frequencies, channel, field
// set); each thread takes a contiguous run of steps, starts every
// frequency's phasor with sincospi at the run's first step and advances it
// by one complex rotation per step, then the CTA sums the runs in a fixed
// tree.  Stage 2 (k_s_assemble): one CTA per field set (excitation): the
// power waves of every channel, the peak of the excited channel's incident
// wave and the ratios.  Everything is float64, as in the reference.
#include "fitb_common.cuh"

#include <cmath>

namespace fitb {

namespace {

constexpr int kFB = 8;           // frequencies per CTA
constexpr int kDftThreads = 256;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// X[(b * nch + c) * nf + f] for V (xv) and I (xi) of channel c, field set b,
// over steps [0, N) of the recorder rows (stride nch, field-set stride cap).
__global__ void __launch_bounds__(kDftThreads)
    k_vi_dft(const double* __restrict__ V, const double* __restrict__ I, long long cap, int nch, long long N,
             const double* __restrict__ f, int nf, double dt, double2* __restrict__ xv, double2* __restrict__ xi) {
    const int fb = blockIdx.x * kFB, c = blockIdx.y, b = blockIdx.z;
    const int nfb = min(kFB, nf - fb);
    const long long run = (N + kDftThreads - 1) / kDftThreads;
    const long long n0 = (long long)threadIdx.x * run, n1 = min(n0 + run, N);
    double2 av[kFB], ai[kFB], ph[kFB], rot[kFB];
#pragma unroll
    for (int q = 0; q < kFB; ++q) {
        av[q] = make_double2(0.0, 0.0);
        ai[q] = make_double2(0.0, 0.0);
        const double fq = q < nfb ? f[fb + q] : 0.0;
        // exp(-2 pi j f n dt) = cos(pi x) - j sin(pi x) with x = 2 f n dt
        double s, co;
        sincospi(2.0 * fq * dt * (double)n0, &s, &co);
        ph[q] = make_double2(co, -s);
        sincospi(2.0 * fq * dt, &s, &co);
        rot[q] = make_double2(co, -s);
    }
    const double* v = V + (long long)b * cap * nch + c;
    const double* iv = I + (long long)b * cap * nch + c;
    for (long long n = n0; n < n1; ++n) {
        const double x = v[n * nch], y = iv[n * nch];
#pragma unroll
        for (int q = 0; q < kFB; ++q) {
            av[q].x += x * ph[q].x;
            av[q].y += x * ph[q].y;
            ai[q].x += y * ph[q].x;
            ai[q].y += y * ph[q].y;
            ph[q] = cmul(ph[q], rot[q]);
        }
    }
    // fixed-order tree over the CTA: warp shuffles, then the warps in order
    __shared__ double red[kDftThreads / 32][4 * kFB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kFB; ++q) {
        double t[4] = {av[q].x, av[q].y, ai[q].x, ai[q].y};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double x = t[k];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) red[warp][4 * q + k] = x;
        }
    }
    __syncthreads();
    if (threadIdx.x < 4 * nfb) {
        double acc = 0.0;
        for (int w = 0; w < kDftThreads / 32; ++w) acc += red[w][threadIdx.x];
        const int q = threadIdx.x >> 2, k = threadIdx.x & 3;
        double2* out = (k < 2 ? xv : xi) + ((long long)b * nch + c) * nf + fb + q;
        reinterpret_cast<double*>(out)[k & 1] = acc;
    }
}

// maps: [nch][4][nf] complex (aV, aI, bV, bI); S: [nf][nch][B]; A: [nf][B].
__global__ void k_s_assemble(const double2* __restrict__ xv, const double2* __restrict__ xi, int nch, int nf,
                             const double* __restrict__ f, double dt, const double2* __restrict__ maps,
                             const int* __restrict__ icot, const int* __restrict__ excited, double thr, int B,
                             double2* __restrict__ S, double2* __restrict__ A) {
    const int b = blockIdx.x;
    const int ex = excited[b];
    __shared__ double s_peak[32];
    // peak |a_excited| over the frequency axis
    double peak = 0.0;
    auto wave = [&](int c, int q, int which) {  // which 0: a, 1: b
        const double2 vf = xv[((long long)b * nch + c) * nf + q];
        double2 cf = xi[((long long)b * nch + c) * nf + q];
        if (!icot[c]) {
            double s, co;
            sincospi(f[q] * dt, &s, &co);  // exp(+j omega dt / 2)
            cf = cmul(cf, make_double2(co, s));
        }
        const double2* m = maps + (long long)c * 4 * nf;
        const double2 kv = m[(2 * which) * nf + q], ki = m[(2 * which + 1) * nf + q];
        const double2 t1 = cmul(kv, vf), t2 = cmul(ki, cf);
        return make_double2(t1.x + t2.x, t1.y + t2.y);
    };
    if (ex >= 0)
        for (int q = threadIdx.x; q < nf; q += blockDim.x) {
            const double2 a = wave(ex, q, 0);
            peak = fmax(peak, hypot(a.x, a.y));
        }
    for (int o = 16; o > 0; o >>= 1) peak = fmax(peak, __shfl_xor_sync(0xffffffffu, peak, o));
    if ((threadIdx.x & 31) == 0) s_peak[threadIdx.x >> 5] = peak;
    __syncthreads();
    if (threadIdx.x == 0) {
        double p = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) p = fmax(p, s_peak[w]);
        s_peak[0] = p;
    }
    __syncthreads();
    peak = s_peak[0];
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int t = threadIdx.x; t < nf * nch; t += blockDim.x) {
        const int q = t / nch, c = t - q * nch;
        double2 out = make_double2(nan, nan);
        if (ex >= 0 && peak > 0.0) {
            const double2 a = wave(ex, q, 0);
            if (hypot(a.x, a.y) >= thr * peak) {
                const double2 bw = wave(c, q, 1);
                const double den = a.x * a.x + a.y * a.y;
                out = make_double2((bw.x * a.x + bw.y * a.y) / den, (bw.y * a.x - bw.x * a.y) / den);
            }
        }
        S[((long long)q * nch + c) * B + b] = out;
        if (A && c == 0) A[(long long)q * B + b] = ex >= 0 ? wave(ex, q, 0) : make_double2(0.0, 0.0);
    }
}

}  // namespace

void launch_vi_dft(const double* V, const double* I, long long cap, int nch, long long N, int B, const double* f,
                   int nf, double dt, double2* xv, double2* xi, cudaStream_t s) {
    if (nf <= 0 || nch <= 0 || B <= 0) return;
    k_vi_dft<<<dim3((nf + kFB - 1) / kFB, nch, B), kDftThreads, 0, s>>>(V, I, cap, nch, N, f, nf, dt, xv, xi);
}

void launch_s_assemble(const double2* xv, const double2* xi, int nch, int nf, const double* f, double dt,
                       const double2* maps, const int* icot, const int* excited, double thr, int B, double2* S,
                       double2* A, cudaStream_t s) {
    if (nf <= 0 || nch <= 0 || B <= 0) return;
    k_s_assemble<<<B, 256, 0, s>>>(xv, xi, nch, nf, f, dt, maps, icot, excited, thr, B, S, A);
}

}  // namespace fitb
