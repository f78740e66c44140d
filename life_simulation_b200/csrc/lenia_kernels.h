// life_simulation_b200/csrc/lenia_kernels.h -- host-side launchers of the
// CUDA kernels (internal interface between the module and the .cu files).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "lenia_types.h"

namespace lenia {

// ----------------------------------------------------------------- direct
enum DirectTileCfg { kDirectTile32x16 = 0, kDirectTile64x16 = 1, kDirectTile64x32 = 2 };

struct DirectGeometry {
    int r;      // halo radius (max kernel radius, integer)
    int ksize;  // 2r + 1 kernel rows
    int xp;     // r rounded up to a multiple of 4
    int wp;     // weight row pitch = 2*xp + 8
};

size_t direct_smem_bytes(int tile_cfg, int nk, const DirectGeometry& g);

// One world of a batched direct launch (single kernel LUT). Its LUT uses the
// world's own geometry g (radius r <= the launch's max_r).
struct DirectWorld {
    const float* src;
    float* dst;
    const float* weights;   // [2r+1][wp]
    const uint32_t* spans;  // [2r+1]
    DirectGeometry g;
    StepParams p;
};
// tiles[i] = (world, tile x, tile y) of 32x16 output tiles.
cudaError_t launch_direct_worlds(const DirectWorld* worlds, const int3* tiles, int ntiles, int max_r,
                                 cudaStream_t stream);
// Halo-tile tensor maps of the direct path: one 2D map per state buffer
// (cuTensorMapEncodeTiled descriptors, opaque here) whose box is a CTA's halo
// tile; `err` counts halo loads whose wait ran out (stays 0 on a healthy
// device).
struct DirectTma {
    alignas(64) unsigned char map[2][128];
    int* err = nullptr;
    bool on = false;
};
// Encodes the maps of fields[0], fields[1] (w x h floats) for the tile shape
// of `tile_cfg`; false (and on = false) when the size cannot use them: width
// not a multiple of 4 floats (16-byte row stride), a halo tile wider or taller
// than the field or than a 256-element box, or no driver entry point.
bool direct_tma_encode(int tile_cfg, const DirectGeometry& g, float* const fields[2], int w, int h, DirectTma& out);
// `tma` (or null): interior tiles load their halo with one TMA box from the
// map of state buffer `buffer` (the one `src` is); edge tiles, whose halo
// wraps around the torus, keep the wrapped element loads.
// `split` (1, or 2/4/8 with 32x16 tiles): kernel rows split over that many
// thread groups per tile, for fields too small to fill the GPU otherwise.
// `ox`: outputs per thread along x (8, or 16 with 64x32 tiles); `oy`: output
// rows per thread (1, or 2 with 64x32 / 64x16 tiles and no split; its
// per-row chunk spans must lie on the 8-tap grid that starts at -xp). The
// same bits in every variant.
cudaError_t launch_direct_step(int tile_cfg, int nk, const float* src, float* dst,
                               const float* weights, const uint32_t* spans,
                               const DirectGeometry& g, const StepParams& p, cudaStream_t stream,
                               const DirectTma* tma = nullptr, int buffer = 0, int split = 1, int ox = 8,
                               int oy = 1);
// Extra shared memory of a split direct launch (the groups' partial sums).
size_t direct_split_smem_bytes(int split, int nk);

// -------------------------------------------------------------------- FFT
constexpr int kMaxPasses = 8;

// A mixed-radix plan for one transform length: n = prod(radix[0..npass)).
struct FftPlan {
    int n;
    int npass;
    int radix[kMaxPasses];
};

// Device geometry of the spectral path for a W x H field (W even).
// Spectra are stored column-major: element (kx, ky) of a plane lives at
// [kx * H + ky], kx in [0, M) with M = W/2; column 0 packs the real DC and
// Nyquist columns as (re, im).
struct FftGeometry {
    int W, H, M;
    FftPlan row;                 // length-M complex transform of a row
    FftPlan col;                 // length-H complex transform of a column
    const float2* tw_row;        // exp(-2 pi i t / M), t < M
    const float2* tw_col;        // exp(-2 pi i t / H), t < H
    const float2* tw_r2c;        // exp(-2 pi i k / W), k <= M
    const float* khat;           // [nk][M + 1][H/2 + 1] real kernel spectra / (W*H)
    int nk;
    int rows_per_cta;            // rows per CTA in the row passes
    int cols_per_cta;            // columns per CTA in the column pass
};

// Row pass: A (H x W) -> spectrum S (M x H column-major, packed column 0).
cudaError_t launch_row_r2c(const FftGeometry& g, const float* A, float2* S, cudaStream_t s);
// Column pass: S -> U_k = IFFT_H(FFT_H(S) * khat_k), k < nk (nk planes).
cudaError_t launch_col_conv(const FftGeometry& g, const float2* S, float2* U, cudaStream_t s);
// Row pass: U_k -> potentials -> growth -> A' (H x W); if S_next is not
// null, also the row spectrum of A' (the next substep's first pass).
cudaError_t launch_row_c2r_growth(const FftGeometry& g, const float2* U, const float* A,
                                  float* A_out, float2* S_next, const StepParams& p,
                                  cudaStream_t s);
size_t fft_row_smem_bytes(const FftGeometry& g);
size_t fft_col_smem_bytes(const FftGeometry& g);

// Compile-time-plan passes (lenia_fft_fast.cu) for the sizes they cover.
// They use the blocked spectral layout: element (kx, ky) of a plane at
// ((kx / kSpectralBlock) * H + ky) * kSpectralBlock + kx % kSpectralBlock
// (M must be a multiple of kSpectralBlock); the runtime-plan kernels above
// use the column-major layout. A context uses one or the other throughout.
constexpr int kSpectralBlock = 8;
struct FastPlan {
    int n = 0;
    int np = 0;
    int radix[kMaxPasses] = {};
};
struct FastTables {
    const float2* col_twf = nullptr;  // column forward plan, per-pass twiddles
    const float2* col_twi = nullptr;  // column inverse plan (reversed passes)
    const float2* row_twi = nullptr;  // row inverse plan
    const float2* row_twf = nullptr;  // row forward plan (reversed passes)
};
// One world of a spectral pass launch. A launch covers one world (passed by
// value) or a table of worlds of the same size (blockIdx.y = world index).
struct ColorMapParams {  // ColorMapParams, Shaders/Render/ColorMap.metal:6-15
    float a[3], b[3], c[3], d[3];
    float input_scale, input_bias, exposure;
    uint32_t channel;
};
struct SpectralWorld {
    const float2* S;     // row spectrum of A (blocked layout)
    float2* U;           // nk potential spectra (blocked layout)
    const float* khat;   // nk kernel spectra, (M+1) x (H/2+1) each
    const float* A;      // state in
    float* A_out;        // state out
    float2* S_next;      // row spectrum of A_out, or null
    float* U_px;         // row pass: nk potential planes (H x W) to keep, or null
    uint2* rgba;         // row pass: the colour layer of A_out (H x W RGBA16F texels), or null
    int M;               // columns of the half spectrum (W/2)
    int nk;              // kernels (0: row pass computes only S_next of A)
    StepParams p;
    ColorMapParams cm;   // palette of `rgba`
};

bool fast_col_plan(int H, FastPlan& forward_plan);
bool fast_row_plan(int M, FastPlan& inverse_plan);
void fast_plan_twiddles(const FastPlan& plan, std::vector<float2>& out);
// The four per-pass twiddle tables of a size's plans, in FastTables order
// (column forward, column inverse, row inverse, row forward); false when H or
// M has no compile-time plan.
bool fast_twiddle_tables(int H, int M, std::vector<float2> (&out)[4]);
// batch: columns per CTA iteration (2, 4 or 8) / rows per CTA iteration
// (1, 2 or 4), for the row pass optionally | kRowPipelined (the variant that
// prefetches the next staged item while transforming the current one; it
// needs a third shared buffer). launch_row_fast with nk = 0 computes only the
// row spectrum of A into S_next (U, A_out unused). The row pass stages A with
// 16-byte copies: A must be 16-byte aligned.
constexpr int kRowPipelined = 0x100;
// Columns per CTA | kHalfThreads (4 only): the column pass with half the
// threads per CTA, each taking two last-pass items (twice the independent
// work per thread).
constexpr int kHalfThreads = 0x40;
// The candidates an autotuner times.
constexpr int kColCandidates[4] = {8, 4, 2, 4 | kHalfThreads};
constexpr int kRowCandidates[6] = {4, 2, 1, 4 | kRowPipelined, 2 | kRowPipelined, 1 | kRowPipelined};
// Whether columns per CTA `col_batch` (8/4/2) and rows per CTA `row_batch`
// (4/2/1, optionally | kRowPipelined) launch for an H x 2M field on the
// compile-time-plan passes (thread count and shared memory within limits).
bool fast_shapes_supported(int H, int M, int col_batch, int row_batch);
cudaError_t launch_col_fast(const FftGeometry& g, const FastTables& t, int batch, const float2* S,
                            float2* U, cudaStream_t s);
cudaError_t launch_row_fast(const FftGeometry& g, const FastTables& t, int batch, const float2* U,
                            const float* A, float* A_out, float2* S_next, const StepParams& p,
                            int nk, cudaStream_t s, void* rgba16f = nullptr, const ColorMapParams* cm = nullptr);
// Many worlds of one size (W = 2M, H) in one launch per pass: `worlds` is a
// device array of n entries; H, M select the compile-time plans. tw_r2c:
// exp(-2 pi i k / W), k <= M (device).
cudaError_t launch_col_fast_worlds(int H, int M, const FastTables& t, int batch,
                                   const SpectralWorld* worlds, int n, cudaStream_t s);
cudaError_t launch_row_fast_worlds(int H, int M, const FastTables& t, const float2* tw_r2c, int batch,
                                   const SpectralWorld* worlds, int n, cudaStream_t s);

// One persistent launch per substep of a batch (lenia_batch_persistent.cu):
// CTAs of kPersistThreads claim work items in list order; a row item waits
// for its world's column items (a counter per world); the last CTA advances
// every world's frame index and substep seed.
constexpr int kPersistThreads = 256;
constexpr int kPersistCtlHead = 32;  // counters per set before the per-world ones
enum PersistKind { kPersistCol = 0, kPersistRow = 1, kPersistDirect = 2 };
struct alignas(16) PersistItem {
    const void* world;     // this parity's SpectralWorld (col/row) or DirectWorld entry
    const float2* tw0;     // column: forward plan twiddles; row: inverse plan twiddles
    const float2* tw1;     // column: inverse plan twiddles; row: forward plan twiddles
    const float2* tw2;     // row: exp(-2 pi i k / W), k <= M
    int kind;              // PersistKind
    int shape;             // column: H; row: M (selects the compiled body)
    int group;             // column: first column; row: first row; direct: tile x | tile y << 16
    int world_id;          // the world's dependency counter
    int need;              // row: column items of the world that precede it
    int count;             // column / row: consecutive groups in this item (from `group` on)
    int pad[2];
};
// Columns (rows) per item of the persistent bodies for a column length H
// (half-spectrum width M); 0 when there is no body for that length.
int persist_col_group(int H);
int persist_row_group(int M);
// Dynamic shared memory of a persistent launch whose items use these column
// lengths, row lengths and direct halo radius (0: no direct items).
size_t persist_smem_bytes(const std::vector<int>& col_h, const std::vector<int>& row_m, int direct_max_r);
// Resident CTAs of the persistent kernel at that shared memory (0 on error).
int persist_grid(size_t smem);
// ctl: 2 counter sets of kPersistCtlHead + nworlds words, zero before the
// first launch; launches alternate par 0/1. loc/base_seed/frame: the batch's
// seed-advance tables (advance = false leaves them, e.g. for timing).
// err: set to 1 when a row item's wait runs out.
cudaError_t launch_persistent(const PersistItem* items, int nitems, uint32_t* ctl, int nworlds, int par,
                              StepParams* const* loc, const uint32_t* base_seed, uint32_t* frame, bool advance,
                              int* err, size_t smem, int grid, cudaStream_t s);

// Column pass with its DFT stages on the tensor cores (lenia_fft_tc.cu), same
// contract and layout as launch_col_fast: precision 1 = BF16 hi/lo, 2 = FP16
// hi/lo operands (FP32 accumulation); H with an all-radix-16 plan (256, 4096);
// batch = columns per CTA iteration (256: 2/4/8, 4096: 1/2).
bool tc_col_plan(int H);
cudaError_t launch_col_tc(const FftGeometry& g, const FastTables& t, int precision, int batch, const float2* S,
                          float2* U, cudaStream_t s);
// The same column pass for H = 4096 with its DFT stages as tcgen05 GEMMs
// (lenia_fft_tc05.cu: two radix-64 passes, operands in shared memory,
// accumulators in tensor memory); same precisions and contract. pipelined:
// two operand slots, so one kernel's MMAs overlap the next kernel's operand
// build. err: device counter of CTAs whose wait for an MMA ran out (or null).
bool tc05_col_plan(int H);
cudaError_t launch_col_tc05(const FftGeometry& g, int precision, bool pipelined, const float2* S, float2* U,
                            int* err, cudaStream_t s);
// Column-pass choices of a context whose column stages run on the tensor
// cores, beside the mma.sync pass's columns-per-CTA counts: the tcgen05 pass,
// serial or pipelined.
constexpr int kTcgen05 = 0x80;
constexpr int kTcgen05Pipelined = 0x81;

// Colour map (lenia_colormap.cu): the field (w x h) to ow x oh RGBA16F
// (ushort4 per pixel); bilinear with wrapping when the sizes differ.
cudaError_t launch_colormap(const float* field, int w, int h, const ColorMapParams& p, void* rgba16f, int ow,
                            int oh, cudaStream_t s);

// ------------------------------------------------------------------ inits
cudaError_t launch_init_noise(float* A, const InitParams& p, cudaStream_t s);
cudaError_t launch_init_stamp(float* A, uint32_t w, uint32_t h, const float* org, uint32_t ow,
                              uint32_t oh, uint32_t count, uint32_t rotate, uint32_t seed,
                              cudaStream_t s);

}  // namespace lenia
