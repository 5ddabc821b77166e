// Internal interface of the learned gauge-covariant preconditioner (kernels in
// learned.cu, solver use in dwf_plan.cu).  Not part of the public C ABI.
#pragma once

#include <cuda_runtime.h>

#include "dwf_kernels.h"

struct b200_dwf;
struct b200_lp;

namespace b200 {

// Paths of one gauge-covariant 5D convolution layer:
//   0 identity, 1 s+1, 2 s-1 (open ends), 3 + 2*mu + {0: +mu, 1: -mu}
// (+mu: U_mu(x) v(x+mu); -mu: U_mu(x-mu)^+ v(x-mu); boundary phase at the edge).
constexpr int kLpPaths = 11;
constexpr int kLpIn = 4;     // channels of the input/output field (the 4 spins)

// Activation layout (f32, one parity): the site-major column of the spinor
// fields with C channels in place of the 4 spins -- 16-byte chunks (k, s) at
// k*Ls + s of the site's column, chunk k holding complex q = 2k, 2k+1 with
// q = color + 3*channel.  For C = 4 this is exactly the f32 spinor layout.
struct LpConvParams {
  const float4* in_same;   // input on the output parity (identity, s paths)
  const float4* in_other;  // input on the other parity (the 8 hop paths)
  float4* out;
  const void* links;       // plan links, f32 two-row records
  const void* links_folded;  // plan links, f32 full records with the boundary phases and
                             // the hop's factor 2 on t links folded in (tensor-core kernel)
  const float2* w;         // [kLpPaths][COUT][CIN] complex weights (BF16 values)
  int* err;                // plan's device error word (bounded waits), or null
  int vh, nx2, ny, nz, nt, ls, ieo;
  float bc[4];
};

struct LpGradParams {
  const float4* delta;     // dL/dy of the layer output (COUT channels)
  const float4* in_same;   // layer input on the output parity (CIN channels)
  const float4* in_other;  // layer input on the other parity
  const void* links;
  float2* partial;         // [gridDim][kLpPaths*COUT*CIN] per-block sums
  int vh, nx2, ny, nz, nt, ls, ieo;
  float bc[4];
};

cudaError_t launch_lp_conv(int cin, int cout, const LpConvParams& p, cudaStream_t st);
// Returns the number of blocks written to p.partial in *nblocks.
cudaError_t launch_lp_gradw(int cin, int cout, const LpGradParams& p, int max_blocks, int* nblocks,
                            cudaStream_t st);

// Internal handle used by the flexible solver: z = N(r) on f32 fields.
int lp_apply_internal(b200_lp* lp, void* z_f32, const void* r_f32, cudaStream_t st);

// Accessors into the operator plan for learned.cu.
int plan_geometry(b200_dwf* op, Geom* g, float bc[4]);
// The plan's device error word, and its synchronising check (B200_ECUDA and
// cleared when a kernel gave up a bounded wait).
int* plan_error_word(b200_dwf* op);
int plan_check_error(b200_dwf* op, cudaStream_t st);
// true when the plan has a halo exchange hook (a rank of a lattice split along t)
bool plan_has_halo(const b200_dwf* op);
int plan_links_f32(b200_dwf* op, const void** links, cudaStream_t st);
int plan_links_f32_folded(b200_dwf* op, const void** links, cudaStream_t st);
// v = DdagD w on FP32 fields of the plan (the operator's own kernels).
int plan_apply_ddagd(b200_dwf* op, void* v, const void* w, cudaStream_t st);

}  // namespace b200
