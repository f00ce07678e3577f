// Sparse (COO / CSF) structures on the device.
#pragma once
#include "common.cuh"

namespace tsr {

// One compressed-sparse-fiber tree in the reference's layout (every fptr
// level holds nnz offsets into the sorted entry list, crates/tenrso-sparse/
// src/csf.rs:193-254), plus the compute side arrays the MTTKRP kernel needs.
struct CsfDev {
  int ndim = 0;
  int mode_order[kMaxModes] = {};
  int64_t shape[kMaxModes] = {};
  int64_t nnz = 0;
  int64_t level_len[kMaxModes] = {};  // fibers per level (level ndim-1: nnz)
  uint32_t* level_ptr[kMaxModes] = {};  // [level_len+1] nnz offsets (levels < ndim-1)
  uint32_t* level_ids[kMaxModes] = {};  // [level_len] mode-index of each fiber
  uint64_t* keys = nullptr;   // sorted mixed-radix keys in mode_order
  float* vals = nullptr;      // sorted values
  // MTTKRP work decomposition: fixed nnz chunks, the level-0 and level-1
  // fiber that holds each chunk's first entry
  int64_t chunk_nnz = 0;
  int64_t n_chunks = 0;
  uint32_t* chunk_root = nullptr;
  uint32_t* chunk_fiber = nullptr;
  std::vector<void*> allocs;
};

}  // namespace tsr

struct tsr_sparse {
  int device = 0;
  int ndim = 0;
  int64_t shape[tsr::kMaxModes] = {};
  int64_t nnz = 0;
  double norm_sq = 0.0;  // sum of squared values (FP64)
  tsr::CsfDev modes[tsr::kMaxModes];  // CSF rooted at each mode
};

namespace tsr {

// Sparse MTTKRP of `sp` rooted at `mode` into d_out (shape[mode] x R fp32).
// The sums accumulate in FP64 in d_acc (shape[mode] x R doubles, zeroed here)
// and are rounded once into d_out. Factors are device pointers (I_m x R).
int launch_mttkrp_csf(tsr_ctx* ctx, cudaStream_t s, const tsr_sparse* sp, const FactorTable& ft,
                      int R, int mode, float* d_out, double* d_acc);
// Shared-memory limits of the CSF kernels (once per process, before capture).
void init_csf_attributes();
void init_hicoo_attributes();
// CooTensor::new's shape and index checks (coo.rs:101-149), tenrso's wording.
int coo_check_shape(int ndim, const int64_t* shape);
int coo_check_bounds(const int64_t* idx, int64_t nnz, int ndim, const int64_t* shape);

}  // namespace tsr
