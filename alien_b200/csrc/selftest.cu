// selftest.cu -- the failure-detection path of the bounded device-side waits,
// exercised without a fault: one thread polls a word that holds the
// sentinel and that nothing ever writes, as a sweep would poll a value whose
// producer is gone.  The wait gives up after its clock budget, sets the
// error flag and returns, the kernel ends, and the host reads the flag: the
// same path that turns a stuck ILU(0) sweep into AB2_ERR_TIMEOUT with the
// context still usable.
#include <chrono>

#include "ab2_internal.cuh"
#include "sentinel.cuh"
#include "tcgen05.cuh"

namespace ab2 {
namespace {

__global__ void k_selftest_wait(const double* word, int* err, double* out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = wait_value(word, err);
}

// The mbarrier form (the learned preconditioner's grid layer): a barrier
// initialised for one arrival that nothing makes; the bounded wait on its
// first phase gives up and the kernel records it.
__global__ void k_selftest_mbar_wait(int* err) {
  __shared__ unsigned long long bar;
  const unsigned a = tc::smem_u32(&bar);
  if (threadIdx.x == 0) {
    tc::mbar_init(a, 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !tc::mbar_wait(a, 0u, kWaitCycles, nullptr)) atomicOr(err, 1);
}

}  // namespace
}  // namespace ab2

using namespace ab2;

extern "C" int ab2_selftest_bounded_wait(ab2_context* ctx, int* expired, double* seconds) {
  if (!ctx || !expired || !seconds) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    double* word = dev_alloc<double>(ctx, 2);
    int* err = dev_alloc<int>(ctx, 1);
    k_fill_bits<<<1, 1, 0, ctx->stream>>>(1, kSentinel, word);
    check_launch(ctx, "selftest_fill");
    AB2_CUDA(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    const auto t0 = std::chrono::steady_clock::now();
    k_selftest_wait<<<1, 32, 0, ctx->stream>>>(word, err, word + 1);
    check_launch(ctx, "selftest_wait");
    int e = 0;
    AB2_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *expired = e;
    dev_free(ctx, word);
    dev_free(ctx, err);
  });
}

extern "C" int ab2_selftest_mbarrier_wait(ab2_context* ctx, int* expired, double* seconds) {
  if (!ctx || !expired || !seconds) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    int* err = dev_alloc<int>(ctx, 1);
    AB2_CUDA(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    const auto t0 = std::chrono::steady_clock::now();
    k_selftest_mbar_wait<<<1, 32, 0, ctx->stream>>>(err);
    check_launch(ctx, "selftest_mbar_wait");
    int e = 0;
    AB2_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *expired = e;
    dev_free(ctx, err);
  });
}

// Host-side fault injection: the nth device allocation from now on fails
// with AB2_ERR_OOM (once); nth = 0 turns it off.  Every creation path must
// then unwind cleanly and the context stay usable.
extern "C" int ab2_context_inject_alloc_failure(ab2_context* ctx, long long nth) {
  if (!ctx || nth < 0) return AB2_ERR_BAD_ARG;
  ctx->alloc_count = 0;
  ctx->fail_alloc_at = nth;
  return AB2_OK;
}
