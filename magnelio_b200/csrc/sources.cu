// TF/SF plane-wave injection (reference: sources/plane_wave.py:709-733).
//
// After the E update every listed E entry gets coef * f(t_E - dt/2 - delay)
// added, after the H update every listed H entry likewise, with t_E = n dt +
// dt and t_H = n dt + dt + dt/2 formed in the reference's order
// (fit_td.py:955-993).  Entries that two face patches share (box edges) keep
// the reference's patch order: the host groups the contributions of one
// entry (CSR: start[u] .. start[u+1]) and one thread adds them in sequence.
// The waveform is evaluated in float64 and rounded to the field dtype
// before the multiply, the product rounded before the add, as the
// reference's array expression does.
#include "fitb_common.cuh"

namespace fitb {

namespace {

__device__ __forceinline__ double wave_at(const PlaneWaveDev& d, double t) {
    if (d.waveform == 0) {
        const double x = t - d.t0;
        return d.amplitude * exp(-(x * x) / d.den);
    }
    return d.amplitude * sin(d.omega * t);
}

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

template <typename T>
__global__ void k_plane_wave(T* field, long long blk, int B, const PlaneWaveDev d, int side,
                             const long long* __restrict__ step) {
    const PlaneWaveSide& s = side == 0 ? d.e : d.h;
    const long long n = *step;
    const double dt = d.dt;
    const double t = (double)n * dt;
    const double t_arg = side == 0 ? (t + dt) - dt / 2 : ((t + dt) + dt / 2) - dt / 2;
    const long long work = (long long)s.n_unique * B;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < work;
         q += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(q / s.n_unique);
        const long long u = q - (long long)b * s.n_unique;
        const double sc = d.scale[b];
        T* f = field + b * blk + s.off[u];
        T v = *f;
        for (int p = s.start[u]; p < s.start[u + 1]; ++p) {
            double w = wave_at(d, t_arg - s.delay[p]);
            if (sc != 1.0) w = sc * w;
            v = v + mul_rn((T)s.coef[p], (T)w);
        }
        *f = v;
    }
}

}  // namespace

template <typename T>
void launch_plane_wave(T* field, long long blk, int B, const PlaneWaveDev& d, int side, const long long* step,
                       cudaStream_t s) {
    const PlaneWaveSide& sd = side == 0 ? d.e : d.h;
    if (sd.n_unique <= 0) return;
    const long long work = (long long)sd.n_unique * B;
    const int threads = 256;
    const long long want = (work + threads - 1) / threads;
    const int blocks = (int)(want < 148 * 8 ? want : 148 * 8);
    k_plane_wave<T><<<blocks, threads, 0, s>>>(field, blk, B, d, side, step);
}
template void launch_plane_wave<float>(float*, long long, int, const PlaneWaveDev&, int, const long long*,
                                       cudaStream_t);
template void launch_plane_wave<double>(double*, long long, int, const PlaneWaveDev&, int, const long long*,
                                        cudaStream_t);

}  // namespace fitb
