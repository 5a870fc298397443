// Host launchers of the fused kernels: shared-memory sizing, the persistent
// grid, and the kernel instance for the plan's layout, scenario groups per
// CTA and factor precision (the instances live in wds_k_*.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "wds_device.cuh"

namespace wds {

size_t state_smem_bytes(const DevNet& n) { return smem_bytes(n); }

namespace {

// CTAs of a persistent launch of B scenarios: one per scenario, at most as
// many as the device keeps resident at once (SMs x CTAs per SM for the
// kernel's threads and shared memory); the CTAs take the scenarios in rounds.
cudaError_t persistent_grid(const void* kern, int threads, size_t smem, int B, int* grid) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (ce == cudaSuccess)
    ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (ce == cudaSuccess && per_sm < 1) ce = cudaErrorInvalidConfiguration;
  *grid = std::max(1, std::min(B, sms * per_sm));
  return ce;
}

template <class Jobs>
size_t multi_smem(const Jobs& jobs) {
  size_t smem = 0;
  for (int p = 0; p < jobs.n; ++p) {
    const auto& J = jobs.j[p];
    if (!J.n.wide)
      smem = std::max(smem, (size_t)J.n.stab_bytes + (size_t)J.groups * (size_t)J.state_bytes);
  }
  return smem;
}

// One persistent single-plan launch of `kern` (arguments: DevNet, DevWork,
// the call's argument block, the per-group state bytes).
template <class Args>
int launch_single(const void* kern, const DevNet& n, const DevWork& w, const Args& a, int B,
                  int groups, void* stream, const char* who, std::string* err) {
  int st = (int)smem_bytes(n);
  const size_t smem = n.wide ? 0 : (size_t)n.stab_bytes + (size_t)groups * st;
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (ce != cudaSuccess) {
    *err = std::string(who) + ": " + cudaGetErrorString(ce);
    return WDS_E_CUDA;
  }
  int grid = 1;
  ce = persistent_grid(kern, 256 * groups, smem, B, &grid);
  if (ce == cudaSuccess) {
    DevNet n_ = n;
    DevWork w_ = w;
    Args a_ = a;
    void* args[] = {&n_, &w_, &a_, &st};
    ce = cudaLaunchKernel(kern, dim3(grid), dim3(256 * groups), args, smem, (cudaStream_t)stream);
  }
  if (ce != cudaSuccess) {
    *err = std::string(who) + " launch: " + cudaGetErrorString(ce);
    return WDS_E_CUDA;
  }
  return WDS_OK;
}

template <class Jobs>
int launch_jobs(const void* kern, Jobs& jobs, int ctas, void* stream, const char* who,
                std::string* err) {
  const size_t smem = multi_smem(jobs);
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (ce == cudaSuccess && ctas > 0) {
    void* args[] = {&jobs};
    ce = cudaLaunchKernel(kern, dim3(ctas), dim3(768), args, smem, (cudaStream_t)stream);
  }
  if (ce != cudaSuccess) {
    *err = std::string(who) + ": " + cudaGetErrorString(ce);
    return WDS_E_CUDA;
  }
  return WDS_OK;
}

}  // namespace

int launch_forward_multi(FwdJobs& jobs, void* stream, std::string* err) {
  int ctas = 0;
  bool fp32 = false;
  for (int p = 0; p < jobs.n; ++p) {
    FwdJob& J = jobs.j[p];
    if (p > 0 && (J.n.fp32 != 0) != fp32) {
      *err = "wds_forward_multi: the plans mix FP32 and FP64 factors";
      return WDS_E_ARG;
    }
    fp32 = J.n.fp32 != 0;
    J.state_bytes = (int)smem_bytes(J.n);
    J.cta0 = ctas;
    ctas += (J.a.B + J.groups - 1) / J.groups;
  }
  return launch_jobs(fp32 ? forward_multi_kernel_f32() : forward_multi_kernel_f64(), jobs, ctas,
                     stream, "wds_forward_multi", err);
}

int launch_adjoint_multi(AdjJobs& jobs, void* stream, std::string* err) {
  int ctas = 0;
  bool fp32 = false;
  for (int p = 0; p < jobs.n; ++p) {
    AdjJob& J = jobs.j[p];
    if (p > 0 && (J.n.fp32 != 0) != fp32) {
      *err = "wds_adjoint_multi: the plans mix FP32 and FP64 factors";
      return WDS_E_ARG;
    }
    fp32 = J.n.fp32 != 0;
    J.state_bytes = (int)smem_bytes(J.n);
    J.cta0 = ctas;
    ctas += (J.a.B + J.groups - 1) / J.groups;
  }
  return launch_jobs(fp32 ? adjoint_multi_kernel_f32() : adjoint_multi_kernel_f64(), jobs, ctas,
                     stream, "wds_adjoint_multi", err);
}

int launch_forward(const DevNet& n, const DevWork& w, const FwdArgs& a, int groups,
                   void* stream, std::string* err) {
  const void* kern = n.fp32 ? forward_kernel_f32(n.wide, groups) : forward_kernel_f64(n.wide, groups);
  return launch_single(kern, n, w, a, a.B, n.wide ? 1 : groups, stream, "wds_forward", err);
}

int launch_unrolled(const DevNet& n, const DevWork& w, const UnrollArgs& u, int plan_groups,
                    void* stream, std::string* err) {
  const int groups = n.wide ? 1 : std::min(plan_groups, 3);  // at most 3 groups per CTA
  const void* kern = n.fp32 ? unrolled_kernel_f32(n.wide, groups) : unrolled_kernel_f64(n.wide, groups);
  return launch_single(kern, n, w, u, u.B, groups, stream, "wds_unrolled_adjoint", err);
}

int launch_adjoint(const DevNet& n, const DevWork& w, const AdjArgs& a, int groups,
                   void* stream, std::string* err) {
  const void* kern = n.fp32 ? adjoint_kernel_f32(n.wide, groups) : adjoint_kernel_f64(n.wide, groups);
  return launch_single(kern, n, w, a, a.B, n.wide ? 1 : groups, stream, "wds_adjoint", err);
}

}  // namespace wds
