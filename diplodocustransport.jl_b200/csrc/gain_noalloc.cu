// dtb_gain_contract_noalloc: the gain contraction of dtb_gain_contract with its scratch in a
// fixed static device array instead of memory allocated by the library.
//
// Some callers cannot call cudaMalloc. A host application that gives all device memory to
// its own pool allocator (a Julia session whose CUDA.jl pool owns the device heap, or a
// serving process that reserved its HBM budget up front) would see a library-side
// cudaMalloc fail or fragment its arena, and a latency-critical loop cannot afford an
// allocator call that may synchronise the device. This entry point allocates nothing: the
// caller passes the inputs and the output in device memory, and the scratch (work table,
// per-unit partial sums, the f1|f2 staging vector and the kernel error flag) lives in
// g_noalloc_scratch below, which every GPU that loads libdtb.so holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "dtb_internal.h"

namespace {

// Stated limits of the static scratch (about 1.4 MB per device).
constexpr int64_t kNoallocMaxUnits = 32768;  // work units (output row x b-range) per call
constexpr int64_t kNoallocMaxVec = 16384;    // n1 + n2 elements staged per call
constexpr size_t kUnitsBytes = (size_t)kNoallocMaxUnits * sizeof(dtb::GainUnit);  // 1 MiB
constexpr size_t kPartBytes = (size_t)kNoallocMaxUnits * sizeof(double);          // 256 KiB
constexpr size_t kVecBytes = (size_t)kNoallocMaxVec * sizeof(double);             // 128 KiB
constexpr size_t kErrOffset = kUnitsBytes + kPartBytes + kVecBytes;
constexpr size_t kScratchBytes = kErrOffset + 256;

// In host code this name is a host-side stand-in, not a device address: only the address
// returned by cudaGetSymbolAddress (taken once per device below) is passed to kernels.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_dev[64] = {};  // device address of g_noalloc_scratch, per device ordinal

}  // namespace

namespace dtb {
// The device address of this entry's kernel error flag on `dev`, or nullptr before the entry's
// set-up on that device (dtb_gain_contract_status reads it).
int* noalloc_flag(int dev) {
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    return g_scratch_dev[dev] ? reinterpret_cast<int*>(static_cast<unsigned char*>(g_scratch_dev[dev]) + kErrOffset)
                              : nullptr;
}
}  // namespace dtb

using namespace dtb;

extern "C" int32_t dtb_gain_contract_noalloc(int32_t dtype, const void* G, int64_t n_out, int64_t n1, int64_t n2,
                                             const void* f1, const void* f2, double* out, void* stream) {
    int rc = gain_op_check_args("dtb_gain_contract_noalloc", dtype, G, f1, f2, out);
    if (rc != DTB_OK) return rc;
    const int esz = dtype == DTB_DTYPE_F64 ? 8 : 4;
    if (n1 <= 0 || n2 <= 0 || n1 + n2 > kNoallocMaxVec) {
        set_error("dtb_gain_contract_noalloc: n1 + n2 must be at most " + std::to_string(kNoallocMaxVec) +
                  " (static scratch limit)");
        return DTB_EINVAL;
    }
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("dtb_gain_contract_noalloc: no current CUDA device");
        return DTB_ENODEV;
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    GainOpPlan plan;
    const int f_len = (int)((n1 + 7) / 8 * 8 + n2);
    rc = gain_op_plan(n_out, n1, n2, esz, sms, gain_stream_blocks_per_sm(esz, f_len), plan);
    if (rc != DTB_OK) return rc;
    if (plan.n_units > kNoallocMaxUnits) {
        set_error("dtb_gain_contract_noalloc: the block needs " + std::to_string(plan.n_units) +
                  " work units; the static scratch holds at most " + std::to_string(kNoallocMaxUnits));
        return DTB_EINVAL;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_dev[dev]) {
            // set-up, once per device, with that device current (the first call on a device)
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                set_error(std::string("dtb_gain_contract_noalloc: cudaGetSymbolAddress failed: ") +
                          cudaGetErrorString(e));
                return DTB_ECUDA;
            }
            g_scratch_dev[dev] = p;
        }
        base = static_cast<unsigned char*>(g_scratch_dev[dev]);
    }
    // The array keeps the previous call's contents. gain_op_run clears the error flag first
    // (in stream order) and then rewrites the work table, the partials and the staged vectors;
    // it places the work table at base, the partials after it (both rounded to 256 bytes) and
    // the staged f1|f2 after those, all within the regions sized above.
    int* err = reinterpret_cast<int*>(base + kErrOffset);
    return gain_op_run(dtype, G, n_out, n1, n2, f1, f2, out, plan, base, err, s);
}
