// Shared device-side definitions of the FIT-TD engine: the padded field
// layout, the per-feature device descriptors, and the launcher prototypes
// implemented in stencil.cu, ports.cu and monitors.cu.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

namespace fitb {

// ---------------------------------------------------------------------------
// Padded uniform layout.
//
// Every one of the six Yee components (and every coefficient array) is
// stored in one common padded box indexed (i, j, k), k fastest:
//   i in [-2, nx+1]  (zero guard planes: two before, one after),
//   j in [0, njp)    with njp = ny + 2,
//   k in [0, nkp)    with nkp = round_up(nz + 2, 8),
// followed by kTailRows zero rows.  A component occupies the sub-box of its
// reference shape; every other entry is a pad that holds +0 forever (its
// update coefficients are 0).  Consequences used by the kernels:
//   * the reference's conditional dual curl ("a missing H neighbour counts
//     as 0", numba_kernels.py:51-58) becomes a plain 4-term stencil, since
//     index j-1 = -1 lands in the previous plane's pad row j = ny+1 and
//     k-1 = -1 in the previous row's pad tail k >= nz+1;
//   * every row starts on a 16-byte boundary (nkp is a multiple of 8: also
//     for the 16-bit compact coefficient copies), and a
//     run of whole rows is one contiguous, 16-byte-aligned byte range: the
//     bulk-copy stencil kernels move row tiles with single cp.async.bulk
//     copies, including one row above the tile (row j0-1 of plane -1 lives
//     in guard plane -2) and up to kTailRows rows past the last plane.
// ---------------------------------------------------------------------------
constexpr int kTailRows = 8;

struct Geom {
    int nx, ny, nz;
    int njp, nkp;
    long long si, sj;  // plane and row strides (elements); sk = 1
    long long vol;     // elements of one padded component
};

__host__ __device__ __forceinline__ long long pidx(const Geom& g, int i, int j, int k) {
    return (long long)(i + 2) * g.si + (long long)j * g.sj + (long long)k;
}

// One CPML face as the stencil kernels see it.  The psi state of all four
// auxiliary components lives in a uniform slab of dims (dI, dJ, dK) =
// (nx+1, ny+1, nz+1) with the face axis replaced by the layer count n; its
// rows are padded to pk = round_up(dK, 16) entries (entry (a, b, c) at
// (a dJ + b) pk + c), so every row starts 16-byte aligned for the air masks
// (bytes) and the psi values alike.  Padding entries hold psi = 0, air = 0.
struct FaceDev {
    int axis;       // 0 = x, 1 = y, 2 = z
    int lo;         // first layer index along the axis
    int n;          // layer count
    int dI, dJ, dK; // slab dims
    int pk;         // row pitch (entries)
    long long slab; // dI * dJ * pk
    void* psi;      // [B][4][slab] field dtype: E1, E2, H1, H2
    void* psi_next; // fused step: the buffer the new psi goes to
    const unsigned char* air;  // [4][slab] 0/1
    const void* bcc;           // [3][n] field dtype: b, c, ck
};

constexpr int kMaxFaces = 6;

template <typename T>
struct StencilArgs {
    Geom g;
    int B;
    T* e;  // [B][3][vol]
    T* h;  // [B][3][vol]
    T* e_next;  // fused step: the buffers the new E and H go to
    T* h_next;
    const T* aE;
    const T* bE;  // [3][vol]
    const T* aH;
    const T* bH;  // [3][vol]
    int nfaces;
    FaceDev f[kMaxFaces];
    int ichunk;  // planes per CTA along i
    // Compact coefficient storage read by the stream kernels (coef_kind 1:
    // float16, 2: bfloat16): cq = {aE, bE, aH, bH}, each [3][vol] of 16-bit
    // values, value = stored * cs[4 * array + component] (cs[4a+3] unused).
    int coef_kind;
    const unsigned short* cq[4];
    float cs[16];
};

constexpr int kCoefNative = 0, kCoefF16 = 1, kCoefBF16 = 2;

// dst[q] = 16-bit(src[q] * inv_scale), round to nearest even.
template <typename T>
void launch_compact(const T* src, unsigned short* dst, long long n, float inv_scale, int coef_kind, cudaStream_t s);

template <typename T>
void launch_update_E(const StencilArgs<T>& a, cudaStream_t s);
template <typename T>
void launch_update_H(const StencilArgs<T>& a, cudaStream_t s);

// Software-pipelined register stencil, batched over B in {1, 2, 4, 8, 16}
// field sets (the default kernels).
struct StreamPlan {
    int ichunk;
    int grid_x, grid_y, grid_z;
    int block_y;  // warp rows per CTA (grid rows x field sets)
};
bool stream_batch_supported(int B);
// variant: register cap (0 natural, 1-3 capped; 2, 3 need B <= 8)
bool stream_variant_supported(int B, int variant);
template <typename T>
int stream_occupancy(int B, int coef_kind, int variant);
StreamPlan plan_stream(const Geom& g, int sm_count, int ctas_per_sm, int B);
// which: 0 = E update, 1 = H update
template <typename T>
void launch_stream_half(StencilArgs<T> a, const StreamPlan& sp, int variant, int which, cudaStream_t s);

// Vectorised stencil over flattened padded planes, batched like the stream
// kernels (B <= 8); grid_y = 1 and block_y is the CTA's warp count.
// variant: vector width x register cap (stencil_vec.cu).
int vec_width_of(int prec, int variant);
template <typename T>
int vec_occupancy(int variant, int coef_kind);
StreamPlan plan_vec(const Geom& g, int sm_count, int ctas_per_sm, int B, int vk);
template <typename T>
void launch_vec_half(StencilArgs<T> a, const StreamPlan& sp, int variant, int which, cudaStream_t s);

// Fused step (E then H in one i-march, stencil_fused.cu): reads e, h, psi
// and writes e_next, h_next, psi_next.  variant: register prefetch with 8 or
// 16 rows per CTA (0, 1) or the cp.async shared-memory pipeline with 3 or 4
// stages (2, 3); block_y = rows per CTA.
int fused_tj_of(int variant);
template <typename T>
cudaError_t prepare_fused(int variant);
template <typename T>
int fused_occupancy(int variant);
StreamPlan plan_fused(const Geom& g, int sm_count, int ctas_per_sm, int B, int tj);
template <typename T>
void launch_fused_step(StencilArgs<T> a, const StreamPlan& sp, int variant, cudaStream_t s);
// TMA-fed shared-memory tile form of the fused step (stencil_tile.cu), the
// fused-step variants kFusedTileBase + v for tile variant v (tile rows, ring
// stages; 32 cells per row): 0 (4, 3), 1 (4, 4), 2 (8, 4), 3 (16, 4),
// 4 (4, 5), 5 (8, 3), 6 (2, 4), 7 (3, 3), 8 (2, 3).  grid_x = k tiles x
// field sets, grid_y = j
// tiles, grid_z = i chunks.  The tile kernel carries no CPML: after it,
// launch_tile_cpml_E applies the E-side CPML face by face to e_next, and
// after the ports' E writes launch_tile_cpml_H recomputes H on every cell
// the CPML reaches.
constexpr int kFusedTileBase = 7, kTileVariants = 9;
template <typename T>
bool tile_supported(int variant);
template <typename T>
cudaError_t prepare_tile(int variant);
template <typename T>
int tile_occupancy(int variant);
template <typename T>
StreamPlan plan_tile(const Geom& g, int sm_count, int ctas_per_sm, int B, int variant);
// Encodes the tensor maps of the current buffers and launches; < 0 when the
// maps cannot be encoded.  status: set non-zero when a bounded wait expires.
template <typename T>
int launch_tile_step(StencilArgs<T> a, const StreamPlan& sp, int variant, int* status, cudaStream_t s);
// Both return the number of launches issued (< 0: a grid too large for
// their 32-bit offsets or more pass boxes than the table holds, which
// tile_step_fits rules out beforehand).
template <typename T>
int launch_tile_cpml_E(const StencilArgs<T>& a, cudaStream_t s);
template <typename T>
int launch_tile_cpml_H(const StencilArgs<T>& a, cudaStream_t s);
// Slab form of the fused step (stencil_slab.cu): the tile march with the
// CPML applied inside it, launched once per list of units with 0..3 CPML
// face slots; fused-step variants kFusedSlabBase + v with (tile rows, ring
// stages of the CPML-free list, of the CPML lists) = (4, 3, 3), (2, 3, 3),
// (3, 3, 3), (4, 4, 4), (3, 4, 4), (2, 4, 4), (8, 3, 3), (6, 3, 3) for
// v = 0..7, one field set per CTA; v = 8, 9: (4, 3, 3) with 2 and 4 field
// sets per CTA sharing the coefficient boxes.
constexpr int kFusedSlabBase = kFusedTileBase + kTileVariants, kSlabVariants = 10;
inline bool is_tile_variant(int v) { return v >= kFusedTileBase && v < kFusedSlabBase; }
inline bool is_slab_variant(int v) { return v >= kFusedSlabBase && v < kFusedSlabBase + kSlabVariants; }
int slab_tj_of(int variant);
int slab_nb_of(int variant);  // field sets per CTA
template <typename T>
bool slab_six_ok(int variant, bool air);  // the six-slot instance exists
template <typename T>
bool slab_supported(int variant);
template <typename T>
cudaError_t prepare_slab(int variant);
template <typename T>
int slab_occupancy(int variant);
template <typename T>
StreamPlan plan_slab(const Geom& g, int sm_count, int ctas_per_sm, int B, int variant);
// Unit lists by face-slot count 0, 1, 2, 3 and 4-6 (int4: k tile, j tile,
// i chunk, packed slot faces); false when the face table is too large.
constexpr int kSlabLists = 5;
bool plan_slab_units(const Geom& g, const FaceDev* f, int nfaces, int tj, int ichunk,
                     std::vector<int4> out[kSlabLists]);
// Dead-unit skipping: flags[u] = 1 for every unit with a live cell (an E
// edge with a nonzero coefficient, an H face that is neither a no-op nor
// curl-dead); and the sync of the skipped units' cells across both buffer
// sets.  Both return the launches issued.
template <typename T>
int slab_unit_liveness(const Geom& g, const T* aE, const T* bE, const T* aH, const T* bH, int tj, int ichunk,
                       const int4* units, int n, int* flags, cudaStream_t s);
template <typename T>
int slab_dead_sync(const Geom& g, const T* aH, const T* bH, int tj, int ichunk, const int4* units, int n, int B,
                   T* e_cur, T* h_cur, T* e_oth, T* h_oth, cudaStream_t s);
// Launches one kernel per non-empty unit list, list q on streams[q] (the
// units are disjoint: the caller may run the streams side by side); returns
// the launches issued (< 0: tensor maps not encodable).  air: some face has
// PEC masks.
template <typename T>
int launch_slab_step(StencilArgs<T> a, int ichunk, int variant, const int4* const units[kSlabLists],
                     const int n_units[kSlabLists], bool air, int* status, const cudaStream_t streams[kSlabLists]);
// One CTA waits, bounded by `limit` tries, on an mbarrier that nothing
// completes; the expired wait writes kStatusWaitTimeoutTile to *status.
cudaError_t launch_wait_probe(int* status, unsigned limit, cudaStream_t s);
// Whether the tile step takes this grid and CPML layout.
template <typename T>
bool tile_step_fits(const StencilArgs<T>& a);
// H update of listed cells (x, y, z = i, j, k) from h / psi and e_next.
template <typename T>
void launch_fix_H(const StencilArgs<T>& a, const int4* cells, int n, cudaStream_t s);

// Bulk-copy (TMA) pipelined stencil kernels for a single field set.
// status: device word set non-zero when a bounded pipeline wait gives up.
struct BulkPlan {
    int tj;        // rows per tile (1 or 2)
    int stages;    // shared-memory ring depth
    int threads;   // CTA size
    int ntiles;    // tiles along j
    int nchunks;   // chunks along i
    int ichunk;    // planes per chunk
    size_t smem;   // dynamic shared memory bytes
};
template <typename T>
BulkPlan plan_bulk(const Geom& g, int sm_count);
// Sets the dynamic shared-memory limit of the bulk kernels (call before any
// capture).
template <typename T>
cudaError_t prepare_bulk(const BulkPlan& plan);
template <typename T>
void launch_update_E_bulk(const StencilArgs<T>& a, const BulkPlan& plan, int* status, cudaStream_t s);
template <typename T>
void launch_update_H_bulk(const StencilArgs<T>& a, const BulkPlan& plan, int* status, cudaStream_t s);
constexpr int kStatusWaitTimeoutE = 1;
constexpr int kStatusWaitTimeoutH = 2;
constexpr int kStatusWaitTimeoutTile = 3;

// ---------------------------------------------------------------------------
// Lumped ports (Thevenin element with a series R-L-C companion).
// ---------------------------------------------------------------------------
struct LumpedDev {
    int n_edges;
    const long long* off;   // [n_edges] offset into the field set's E block
    const double* sign;     // [n_edges]
    const double* beta;     // [n_edges]
    double beta_sum;
    double R, L, C;         // < 0: absent
    double rec_scale;
    const double* src;      // [B][n_src]
    long long n_src;
    double* st;             // [B][4]: i_prev, vL, vC, last_I
    int channel;            // recorder channel
};

// ---------------------------------------------------------------------------
// Modal ports (projection, modal Mur / TF-SF, exact DTBC, reconstruction,
// complement absorber, V/I recording).
// ---------------------------------------------------------------------------
constexpr int kMaxModes = 16;

struct ModalDev {
    int n_modes;
    int n_e, n_e_u;   // port-plane E samples (u + v), u count
    int n_h, n_h_u;
    const long long* port_e;  // [n_e] offsets into the E block
    const long long* int_e;   // [n_e]
    const long long* port_h;  // [n_h] offsets into the H block
    const double* me_port;    // [n_e]
    const double* me_int;     // [n_e]
    const double* mh_port;    // [n_h]
    const double* eprof;      // [M][n_e]
    const double* vprof;      // [M][n_e]
    const double* hprof;      // [M][n_h]
    double mur_r[kMaxModes];
    double tau[kMaxModes];
    double rec_scale[kMaxModes];
    int is_dtbc[kMaxModes];
    double r2[kMaxModes], q2[kMaxModes];
    // DTBC kernels: per mode, the concatenation of the tables of length
    // n0, 2 n0, 4 n0, ... (n_tables of them).
    const double* ktab[kMaxModes];
    int n0;
    int n_tables;
    int comp_on;
    const double* comp_r;     // [n_e]
    const double* comp_live;  // [n_e]
    // per field set state and sources
    double* st;               // [B][ST_SIZE] scalars (see ports.cu)
    double* whist;            // [B][M][cap]
    double* shist;            // [B][M][cap]
    double* comp_state;       // [B][2][n_e] complement int_prev, port_prev
    double* scratch;          // [B][2][n_e] gathered interior samples, new plane values
    const int* exc_mode;      // [B] excited mode or -1
    const double* wf;         // [B][n_wf] waveform(n dt)
    long long n_wf;
    const int* buf_len;       // [B] TF/SF source buffer length
    long long cap;            // history capacity (steps)
    int channel0;             // first recorder channel
    double dt;
    // DTBC convolution partial sums of the current step, per history chunk
    // of kConvChunk entries: [B][M][conv_chunks][2] (w, s)
    double* conv;
    int conv_chunks;
    // large planes (n_chunks > 1): the projections and the reconstruction
    // run over n_chunks CTAs of `chunk` edges and faces each (ports.cu)
    int n_chunks, chunk;
    double* part;  // [B][n_chunks][2 kMaxModes] projections, then [B][n_chunks][kMaxModes] V sums
    double* vals;  // [B][2 kMaxModes]: the step's boundary values and interior projections
    int* done;     // [B] reconstruction CTAs finished this step (the last one resets it)
};

constexpr int kPortChunk = 1024;  // edges per CTA of a large plane

constexpr int kConvChunk = 1024;

struct RecorderDev {
    double* V;  // [B][cap][nch]
    double* I;  // [B][cap][nch]
    int nch;
    long long cap;
};

struct PortsArgs {
    int B;
    long long e_block;  // elements per field set (3 * vol)
    long long h_block;
    const long long* step;  // device step counter (completed steps)
    double dt_lumped;       // solver time step
    RecorderDev rec;
    double* absmax;  // [B]
};

template <typename T>
void launch_lumped(T* e, const PortsArgs& pa, const LumpedDev* d, int n_lumped, cudaStream_t s);
// max_chunks: the largest n_chunks of the ports (1: every port in one CTA
// per field set)
template <typename T>
void launch_modal(T* e, const T* h, const PortsArgs& pa, const ModalDev* d, int n_modal, int max_chunks,
                  cudaStream_t s);
// Band-subspace DTBC port (ports_band.cu; ports/_modal/band_dtbc.py): the
// projected boundary period of p <= kBandPMax coordinates with matrix DTBC
// kernels.  Offsets are padded-layout entries of a field set's E (H) block.
constexpr int kBandPMax = 32;
struct BandDev {
    int p, M, channel0, has_in;
    long long n_u, n_v, n1, n_h;
    const long long *eu, *ev, *x1, *hh;       // port plane E (u, v), first interior period, dual H
    const double *Wu, *Wv;                    // [n_u][p], [n_v][p]
    const double *Mc;                         // [p][n1]
    const double *D0, *Dm1;                   // [p][p]
    const double *me, *vprof, *mh, *hprof;    // [n_u + n_v], [M][n_u + n_v], [n_h], [M][n_h]
    const double* rec_scale;                  // [M]
    long long n0;                             // initial kernel length; table t has n0 2^t entries
    const double *kout, *kin;                 // tables one after the other: [L][p][p]
    double* st;                               // [B][2 p]: xt, xt_prev
    double* x1prev;                           // [B][n1]
    double *whist, *shist;                    // [B][cap][p]
    long long cap;
    const double* src;                        // [B][n_src][p]
    long long n_src;
    const int* src_on;                        // [B]
    double* conv;                             // [B][conv_chunks][2][p] partial sums of the step
    int conv_chunks;
};
template <typename T>
void launch_band(T* e, const T* h, const PortsArgs& pa, const BandDev* d, int n_band, int max_chunks, cudaStream_t s);

// The DTBC history convolutions of the coming port update (they read only
// the history before the current step), spread over the history chunks of
// every (port, field set); launch_modal sums the partials in chunk order.
// max_chunks = the largest conv_chunks of the ports.
void launch_dtbc_conv(const PortsArgs& pa, const ModalDev* d, int n_modal, int max_chunks, cudaStream_t s);

// ---------------------------------------------------------------------------
// TF/SF plane waves: per side (E, H) the unique corrected entries (offsets
// into a field set's block) with their contributions in patch order.
// ---------------------------------------------------------------------------
struct PlaneWaveSide {
    long long n_unique;
    const long long* off;   // [n_unique]
    const int* start;       // [n_unique + 1] into coef / delay
    const double* coef;     // field-dtype values held as double
    const double* delay;    // seconds
};

struct PlaneWaveDev {
    int waveform;           // 0 gaussian, 1 sine
    double amplitude, t0, den, omega, dt;
    const double* scale;    // [B]
    PlaneWaveSide e, h;
};

// side 0: after the E update (field = E), 1: after the H update (field = H).
template <typename T>
void launch_plane_wave(T* field, long long blk, int B, const PlaneWaveDev& d, int side, const long long* step,
                       cudaStream_t s);

// ---------------------------------------------------------------------------
// ADE dispersion of one side (dispersion.cu).  States of all blocks are
// concatenated; a state's pole states live at J[b][slot[s] + 2 q'] (real
// part, imaginary part; real poles use the first).
// ---------------------------------------------------------------------------
struct DispDev {
    long long n_states;
    const long long* off;        // [n_states] entry offset in a field set's block
    const void* g;               // [n_states] field dtype
    const int* state_block;      // [n_states]
    const long long* slot;       // [n_states] into a field set's J
    long long n_slots;           // J entries per field set
    void* J;                     // [B][n_slots] field dtype
    void* fprev;                 // [B][n_states] field dtype
    const int* pole_start;       // [n_blocks + 1]
    const int* kind;             // [n_poles] 0 real, 1 conjugate pair
    const double *k_re, *k_im, *c_re, *c_im, *opk_re, *opk_im, *hw;  // [n_poles]
    long long n_unique;          // distinct entries
    const long long* uoff;       // [n_unique]
    const int* ustart;           // [n_unique + 1] into ustate
    const long long* ustate;     // states of each entry, block order
};

template <typename T>
void launch_disp_save(const T* F, long long blk, int B, const DispDev& d, cudaStream_t s);
template <typename T>
void launch_disp_update(T* F, long long blk, int B, const T* beta, const DispDev& d, cudaStream_t s);
// Surface-impedance walls on the H faces (sibc.cu; solver/_sibc.py).
struct SibcDev {
    long long n_states;          // faces of all walls
    const long long* off;        // [n_states] H entry offset in a field set's block
    const void* g;               // [n_states] field dtype
    const int* state_block;      // [n_states] wall of the face
    const long long* slot;       // [n_states] first branch state in a field set's u
    long long n_slots;           // branch states per field set
    void* u;                     // [B][n_slots] field dtype
    void* hprev;                 // [B][n_states] field dtype
    const int* br_start;         // [n_blocks + 1] into the branch tables
    const double *k, *q, *hopk;  // [n_branches]: k, q, (1 + k) / 2
    long long n_unique;          // distinct faces
    const long long* uoff;       // [n_unique]
    const int* ustart;           // [n_unique + 1] into ustate
    const long long* ustate;     // faces of each entry, wall order
};

template <typename T>
void launch_sibc_save(const T* h, long long blk, int B, const SibcDev& d, cudaStream_t s);
template <typename T>
void launch_sibc_update(T* h, long long blk, int B, const T* beta, const SibcDev& d, cudaStream_t s);

// CPML face q of the stencil args as a separate pass; side 0 = E, 1 = H.
template <typename T>
void launch_cpml_pass(const StencilArgs<T>& a, int q, int side, cudaStream_t s);

// ---------------------------------------------------------------------------
// Running-DFT monitors, staged in blocks of K recorded samples.
// ---------------------------------------------------------------------------
struct DftDev {
    int i0, j0, k0, ni, nj, nk;
    long long ncell;
    int ncomp;
    int comps[6];
    int nf;
    const double* omega;  // [nf]
    int stride;
    int kahan;
    int K;
    const long long* base;  // device: first step from which slots are counted
    const double* inv;    // [3][max(nx,ny,nz)+1] primal widths dx,dy,dz and
    const double* dual;   // [3][max+1] solver dual widths
    int inv_ld;           // leading dimension of inv/dual
    float* stage;         // [B][K][ncomp][ncell]
    float2* wst;          // [K][2][nf] phasor weights (E time, H time)
    float2* bins;         // [B][ncomp][nf][ncell]
    float2* cmp;          // Kahan compensation, same shape
    double dt;
    int sblk0, sblk;      // this monitor's blocks in the merged stage launch
    int fblk0, fblk;      // and in the merged flush launch
};

int dft_blocks(long long work);
// One launch stages every monitor; one launch flushes every full monitor and
// advances the step counter (its last CTA, through `ticket`).
template <typename T>
void launch_dft_stage_all(const T* e, const T* h, long long e_block, long long h_block, const Geom& g, int B,
                          const DftDev* devs, int nmon, int nblocks, const long long* step, cudaStream_t s);
void launch_dft_flush_all(int B, const DftDev* devs, int nmon, int nblocks, size_t smem, long long* step,
                          unsigned* ticket, cudaStream_t s);
// Host-requested flush of the first kc slots of one monitor.
void launch_dft_flush_forced(int B, const DftDev& d, int kc, cudaStream_t s);

// Modal S-parameters from the recorder (sparams.cu): the direct DFT of every
// field set's V and I channels over steps [0, N), then the power-wave split
// and S = b / a_excited per field set (excitation).
void launch_vi_dft(const double* V, const double* I, long long cap, int nch, long long N, int B, const double* f,
                   int nf, double dt, double2* xv, double2* xi, cudaStream_t s);
void launch_s_assemble(const double2* xv, const double2* xi, int nch, int nf, const double* f, double dt,
                       const double2* maps, const int* icot, const int* excited, double thr, int B, double2* S,
                       double2* A, cudaStream_t s);

// Material matrices and leapfrog coefficients from the grid and the cell
// materials (setup.cu): writes alpha/beta E and H, M_eps, M_mu into the
// padded arrays and the per-component max |coefficient| into coef_max[4][3].
template <typename T>
void launch_setup_materials(const Geom& g, const double* dx, const double* dy, const double* dz, const int* mat,
                            const double* eps_r, double dt, long long n_cat1, const long long* cat1_idx,
                            const double* cat1_eps, long long n_pec, const long long* pec_idx, T* aE, T* bE, T* aH,
                            T* bH, T* meps, T* mmu, double* coef_max, cudaStream_t s);

// DTBC kernel table on the device (setup.cu): l_m, m < n, of the outgoing
// root lambda(z) of the discrete Klein-Gordon chain with parameters r, q;
// x is scratch of 8 n complex samples.
void launch_dtbc_kernel(double r, double q, int n, double2* x, double* l, cudaStream_t s);

// Lowest n_modes eigenpairs above threshold of K v = lambda M v (K CSR on
// the device, M its diagonal) in float64 (modes.cu); eigenvectors with
// v^T M v = 1 into vec_out [n_modes][n] (host); 0 on success.
int mode_eigensolve(long long n, const long long* rp, const long long* col, const double* val, const double* m,
                    int n_modes, double threshold, double* lam_out, double* vec_out, cudaStream_t s);

// Lowest n_modes eigenpairs of the symmetric positive semi-definite CSR
// matrix L (on the device) orthogonal to the n_null orthonormal vectors Z
// (device, [n_null][n]), by Chebyshev-filtered subspace iteration in float64
// (modes_sparse.cu); b bounds the spectrum; converged when every wanted
// residual is below tol b.  Vectors into vec_out [n_modes][n] (host).
// 0 on success, -1 arguments, -2 CUDA, -4 not converged, -5 rank loss.
int sparse_lowest_eigs(long long n, const long long* rp, const long long* col, const double* val, int n_null,
                       const double* Z, int n_modes, double tol, double b, double* lam_out, double* vec_out,
                       double* res_out, int* iters_out, cudaStream_t s);

// lambda_max of the live leapfrog update operator D^-1/2 C^T M_mu^-1 C D^-1/2
// by a float64 Lanczos iteration (spectral.cu); 0 on success.
template <typename T>
int spectral_lambda(const Geom& g, const T* meps, const T* mmu, const T* bE, int max_iter, double tol, double* lambda,
                    int* iters, cudaStream_t s);

// Energy: per field set 0.5 (sum m_eps e^2 + sum m_mu h^2) in float64.
template <typename T>
void launch_energy(const T* e, const T* h, const T* meps, const T* mmu, const Geom& g, int b,
                   long long e_block, double* partials, int nblocks, double* out,
                   cudaStream_t s);

void launch_advance(long long* step, cudaStream_t s);

// Layout conversion between the reference flat layout and the padded box.
template <typename T>
void launch_pack(const T* flat, T* padded, const Geom& g, int comp, long long flat_off,
                 cudaStream_t s);
template <typename T>
void launch_unpack(const T* padded, T* flat, const Geom& g, int comp, long long flat_off,
                   cudaStream_t s);

// Reference shapes of component c (0..5 = Ex,Ey,Ez,Hx,Hy,Hz).
__host__ __device__ __forceinline__ void comp_shape(const Geom& g, int c, int& ni, int& nj,
                                                    int& nk) {
    ni = g.nx + ((c == 1 || c == 2 || c == 3) ? 1 : 0);
    nj = g.ny + ((c == 0 || c == 2 || c == 4) ? 1 : 0);
    nk = g.nz + ((c == 0 || c == 1 || c == 5) ? 1 : 0);
}

}  // namespace fitb
