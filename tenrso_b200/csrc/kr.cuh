// Khatri-Rao row generation shared by the dense MTTKRP kernels.
//
// Row j of KR = U_{o0} (.) U_{o1} (.) ... (.) U_{o_last} (the factors of all
// modes except `mode`, FORWARD order) is prod_p U_{o_p}[i_p, :] where
// j = ((i_0 * I_{o1} + i_1) * I_{o2} + i_2) ... — the last other mode varies
// fastest, matching the reference's unfold column order (mttkrp.rs:182-240)
// and mttkrp_fused's index extraction (mttkrp.rs:851-870). Rows are formed
// on the fly and never written to HBM.
#pragma once
#include "common.cuh"

namespace tsr {

struct KRSpec {
  int n_other;
  int R;                               // factor row length (row stride)
  uint32_t size[kMaxModes];            // I_{o_p}
  const float* __restrict__ f[kMaxModes];  // U_{o_p}, row-major I x R
};

inline KRSpec make_krspec(const Unfolding& u, const FactorTable& ft, int R) {
  KRSpec s{};
  s.n_other = u.n_other;
  s.R = R;
  for (int p = 0; p < u.n_other; ++p) {
    s.size[p] = (uint32_t)u.other_size[p];
    s.f[p] = ft.ptr[u.other_mode[p]];
  }
  return s;
}

// Decompose unfolding column j into per-mode row offsets (in elements).
__device__ __forceinline__ void kr_row_offsets(const KRSpec& s, uint32_t j, uint32_t* off) {
#pragma unroll
  for (int p = kMaxModes - 1; p >= 0; --p) {
    if (p < s.n_other) {
      uint32_t sz = s.size[p];
      uint32_t q = j / sz;
      off[p] = (j - q * sz) * (uint32_t)s.R;
      j = q;
    }
  }
}

// Mixed-radix position of an unfolding column: idx[p] is the row of factor
// U_{o_p} for the first NO other modes (NO >= the tensor's n_other).
// Decomposed with divisions once; afterwards advanced by small steps whose
// carries are resolved by subtraction (no division, no if-converted divide
// sequences in the unrolled hot loop).
template <int NO>
struct KRCounter {
  uint32_t idx[NO];

  __device__ __forceinline__ void init(const KRSpec& s, uint32_t j) {
#pragma unroll
    for (int p = NO - 1; p >= 0; --p) {
      idx[p] = 0;
      if (p < s.n_other) {
        const uint32_t q = j / s.size[p];
        idx[p] = j - q * s.size[p];
        j = q;
      }
    }
  }

  __device__ __forceinline__ void advance(const KRSpec& s, uint32_t d) {
#pragma unroll
    for (int p = NO - 1; p >= 0; --p) {
      if (p < s.n_other && d != 0) {
        uint32_t v = idx[p] + d;
        uint32_t carry = 0;
        while (v >= s.size[p]) {
          v -= s.size[p];
          ++carry;
        }
        idx[p] = v;
        d = carry;
      }
    }
  }
};

// KR[j, c] for one column c given precomputed row offsets.
__device__ __forceinline__ float kr_value(const KRSpec& s, const uint32_t* off, int c) {
  float v = __ldg(s.f[0] + off[0] + c);
#pragma unroll
  for (int p = 1; p < kMaxModes; ++p)
    if (p < s.n_other) v *= __ldg(s.f[p] + off[p] + c);
  return v;
}

}  // namespace tsr
