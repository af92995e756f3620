// adf_internal.h -- structures shared by the host runtime and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace adf {

// ---- HBM layout of one solve ----------------------------------------------
// field : [2 buffers][4 channels P,Vx,Vy,Vz][nz][ny][nxp] Float32, x fastest.
//         nxp = row pitch (multiple of 4 floats so rows are 16-B aligned).
//         Step `it` reads buffer (it - it_first) & 1 and writes the other.
// mask  : [nz][ny][mw] uint32, one nibble per cell (bit0 P, bit1 Vx,
//         bit2 Vy, bit3 Vz open), cell x in word x/8, nibble x%8.
// psi_p[a]: p-side CPML memory of axis a, [2 buffers][2 sides][...]:
//         a=0: [nz][ny][npml]   a=1: [nz][npml][nxp]   a=2: [npml][ny][nxp]
// psi_v[a]: v-side, the same with npml+1.
// traces: src/rec/vn_src/vn_rec [nt][ntx] (transceiver fastest).
// Staged planes of the step kernel: x range xb-4 .. xb+kXT+3 of a 64-cell
// tile (the halo column xb-1 and Vx at xb+64 included), rows j0-1 .. j0+ty.
constexpr int kStageW = 72;
constexpr int kStepRing = 2;  // the stage of plane k in use while k+1 lands

enum : int {
  SF_MASK = 1,      // solve has a scatterer mask
  SF_PCPML = 2,     // p-side CPML active (npml>1, or npml>=1 with a mask)
  SF_VCPML = 4,     // v-side CPML active (npml>=1)
  SF_FP32 = 8,      // Float32 arithmetic instead of Float64 intermediates
  SF_GF = 32,       // in-loop GF extrapolation between v2vn and vn2v
  SF_GF_TC = 64,    // its far lags on the tensor cores (TF32 split, gf_tc)
};

// Steps per block of the in-loop GF extrapolation: lags older than the block
// are summed once per block, the rest step by step.
constexpr int kGfBlock = 32;
constexpr int kGfRing = 64;  // input-history rows kept receiver-major (>= kGfBlock + 1)

// GF map kinds, as ADF_GF_* in include/adfdtd.h
enum : int { ADF_GF_PV_FROM_PIN_ = 0, ADF_GF_P_FROM_PIN_ = 1, ADF_GF_PV_FROM_PV_ = 2 };

struct SolveDev {
  int nx, ny, nz, nxp;
  int ty, nty;       // tile rows, number of y tiles
  int npml, flags;
  int nt;            // dom.nt
  int it_base;       // 1-based step executed by launch-step 0 of a chunk
  int it_stop;       // last step (inclusive) to execute
  int it_first;      // step whose input field sits in buffer 0
  int ntx, mw;
  int src_ntx;            // columns of src[] (transceivers that inject)
  // x-slab psi rows, quad-aligned: side 0 holds cell x at x, side 1 at
  // x - xs1 (xs1p = (nx-npml) & ~3, xs1v = (nx-npml-1) & ~3), so that a quad's
  // memory is one aligned float4 per side; npp, nvp: the row pitch
  int npp, nvp;
  int xs1p, xs1v;
  double fq, fv, rdx, rdy, rdz;
  float fqf, fvf, rdxf, rdyf, rdzf;
  float* field;
  // four CUtensorMaps (128 B each) over the field: per buffer 0, 1 one with
  // box (kStageW, ty + 2, 1, 3) (P, Vx, Vy of a plane) and one with box
  // (kStageW, ty + 2, 1, 1) (Vz); 4D (x: nxp, y: ny, z: nz, channel: 4),
  // zero fill outside the grid
  const void* fmap;
  long long buf_stride;   // floats per field buffer (4*nz*ny*nxp)
  long long chan_stride;  // floats per channel (nz*ny*nxp)
  float* psi_p[3];
  float* psi_v[3];
  long long psi_p_buf[3], psi_v_buf[3];  // floats per psi buffer
  long long psi_p_side[3], psi_v_side[3];
  const float* coef;      // a_l a_r a_hl a_hr b_l b_r b_hl b_hr (Float32)
  // injection / recording entries, grouped by (y tile, plane, channel)
  const int* tp_off;      // nty*nz*4 + 1 offsets into seg
  const int4* seg;        // {cell (row*nxp + x), first entry, count, 0}
  const float* ent_w;
  const int* ent_tx;      // src column of the entry's transceiver, -1: no source
  const int* ent_slot;    // contribution slot (c*ntx+tx)*8+corner or -1
  float* contrib;         // [4][ntx][8]
  const unsigned char* inb;  // [4][ntx] stencil in bounds
  float* src[4];          // [nt][src_ntx]
  float* rec[4];          // [nt][ntx]; rec[1..3] may be NULL (not kept)
  float* vn_src;          // [nt][ntx] or NULL (no vn2v)
  float* vn_rec;
  const float* dir;       // [ntx][4]
  const uint32_t* mask_bits;  // [nz][ny][mw] or NULL
  int* err;               // per-solve error word
  int pad_;
  // in-loop GF extrapolation, SF_GF only
  const float* gf_t[4];   // (nt_gf, n1, n2) column-major tensors of the map kind
  const int* gf_isrc;     // [n_out] 0-based transceiver columns driven
  const int* gf_irec;     // [n_in] 0-based transceiver columns read
  double* gf_pin;         // [n_in][nt] (p_rec - z0 vn_rec)/2 of recorded rows
  double* gf_part;        // [n_out][gf_ks][2] partial sums of the split reduction
  double* gf_far;         // [n_out][gf_rs][kGfBlock][2] far-lag partials of the current
                          // block of steps, or NULL (the map is summed step by step)
  const float* gf_near;   // [2][n_out][gf_nl][n_in] lags 0..gf_nl-1 of the two tensors,
                          // receiver fastest (blocked kinds), or NULL
  double* gf_ring;        // [kGfRing][n_in] the last input-history rows, row mod kGfRing
  const int* gf_col;      // [ntx] 1 + the last driven source writing the column, 0: none
  double gf_z0;
  int gf_kind, gf_nt, gf_n1, gf_n2;
  int gf_nout, gf_nin;
  int gf_ks;              // receiver splits per driven source (per-step kernel)
  int gf_rs;              // receiver splits of the far-lag kernel, 0 = no blocking
  int gf_nl;              // lags held in gf_near: min(kGfBlock, nt_gf)
  int gf_tc_nch;          // 16-lag chunks of gf_tc
  const float* gf_tc;     // SF_GF_TC: the two tensors packed as tensor-core operand tiles
                          // [n_in][gf_tc_nch][128-source tiles][2][16 lags x 128 sources]
};

// work item: {solve index, y tile | x tile << 16, z0, z1}
struct StepParams {
  SolveDev* solves;
  const int4* items;
  int n_items;
  int step;  // launch-step index within the chunk
};

struct EpiParams {
  SolveDev* solves;
  int n_solves;
  int step;
};


// launch helpers implemented in fdtd_kernels.cu
// one CTA per work item, blockDim (32, max_ty + 1); max_ty <= step_max_ty()
cudaError_t launch_step(const StepParams& p, int grid, int max_ty, cudaStream_t s);
int step_max_ty();
int step_x_tile();  // cells per x tile of a step work item
cudaError_t step_ctas_per_sm(int* n);  // resident step-kernel CTAs per SM (occupancy)
cudaError_t launch_epilogue(const EpiParams& p, int max_ntx, cudaStream_t s);
cudaError_t launch_gf_extrapolate(const EpiParams& p, int max_blocks, int max_nsrc, bool reduce,
                                  cudaStream_t s);
// far-lag part of the in-loop GF extrapolation for the block of kGfBlock steps
// that starts at launch-step p.step
cudaError_t launch_gf_near_pack(const SolveDev& d, float* near, cudaStream_t s);
cudaError_t launch_gf_far(const EpiParams& p, int max_blocks, int max_nsrc, cudaStream_t s);
// the same on the tensor cores for SF_GF_TC solves (gf_tc_kernel.cu): blocks =
// 128-source tiles x gf_rs; launch_gf_far's combine step then adds the splits
cudaError_t launch_gf_far_tc(const EpiParams& p, int max_blocks, cudaStream_t s);
cudaError_t launch_gf_tc_pack(const SolveDev& d, float* out, cudaStream_t s);
int64_t gf_tc_chunks(int64_t nt_gf);  // 16-lag chunks of lags 1 .. nt_gf-1
size_t gf_tc_packed_floats(int64_t nt_gf, int64_t n_src, int64_t n_rec);
int gf_tc_sources_per_tile();

}  // namespace adf
