// Kernels of the plain (single-instance) explicit Euler step, FP64 or FP32.
//
// One step is two launches,
//   gain_stream  - streams the gain blocks G[a][b][c] from HBM through a bulk-copy (TMA)
//                  pipeline in shared memory and contracts each tile against f_b f_c formed
//                  on the fly; writes one FP64 partial per (row, b-range) work unit.
//   euler_rows   - one warp per state row: banded flux row (ELL, 128-bit loads), emission
//                  row pieces, loss bilinear term, sum of the row's gain partials, then the
//                  Euler update and clamp of SteppingMethods.jl:46-101; each block writes a
//                  record of its rows' CFL diagnostics.
// and, once per sequence of steps (a graph of them, or the steps run outside one),
//   step_diag    - one block per step reduces the step's block records (SteppingMethods.jl:48-94)
//                  and advances the step counter, off the steps' critical path.
// The state is double-buffered (f_in -> f_out) because a row reads other rows' f.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "dtb_internal.h"
#include "pdl.cuh"

namespace dtb {

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity; gives up after kWaitLimitNs or when another
// role of the block raised the abort flag.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
        if (globaltimer() - t0 > kWaitLimitNs) return false;
    }
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Julia's min on Float64 with -0.0 ordered below +0.0 (NaN is mapped to Inf before).
__device__ __forceinline__ double jl_min(double a, double b) {
    if (a < b) return a;
    if (b < a) return b;
    return signbit(a) ? a : b;
}
__device__ __forceinline__ double nan_to_inf(double x) { return isnan(x) ? CUDART_INF : x; }

// Julia `x * b::Bool` = ifelse(b, x, copysign(0, x)).
template <typename T>
__device__ __forceinline__ T jl_mul_bool(T x, bool b) {
    return b ? x : copysign(T(0), x);
}

// ------------------------------------------------------------------ gain_stream
struct SpOff {
    int n;
    int off[DTB_MAX_SPECIES + 1];   // unpadded
    int offp[DTB_MAX_SPECIES + 1];  // padded (multiples of 8)
};

template <typename T>
struct Vec;
template <>
struct Vec<float> {
    using type = float4;
    static constexpr int n = 4;
    __device__ __forceinline__ static float dot(const float4& a, const float4& b) {
        return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
    }
};
template <>
struct Vec<double> {
    using type = double2;
    static constexpr int n = 2;
    __device__ __forceinline__ static double dot(const double2& a, const double2& b) {
        return a.x * b.x + a.y * b.y;
    }
};

constexpr int kGainThreads = (kGainConsumerWarps + 1) * 32;

__host__ __device__ constexpr int round_up_int(int x, int m) { return (x + m - 1) / m * m; }

// Reduction ring: a consumer warp can run at most kGainStages tiles (hence units) ahead of
// warp 0, so kGainStages + 2 slots never alias a slot warp 0 is still reading.
constexpr int kRedRing = kGainStages + 2;

int gain_stream_smem_bytes(int elem_size, int f_smem_len) {
    return kGainStages * kGainTileBytes + round_up_int(f_smem_len * elem_size, 16) + 2 * kGainStages * 8 +
           kRedRing * 8 + kRedRing * kGainConsumerWarps * 8 + 16;
}

template <typename T>
__global__ void __launch_bounds__(kGainThreads) gain_stream_kernel(const T* __restrict__ G,
                                                                   const GainUnit* __restrict__ units,
                                                                   int n_units, const T* __restrict__ f,
                                                                   int n_mom, SpOff so, int f_len,
                                                                   double* __restrict__ partial, int* err,
                                                                   const int* __restrict__ cell_list) {
    using V = Vec<T>;
    using vec_t = typename V::type;
    constexpr int kTileElems = kGainTileBytes / sizeof(T);
    constexpr int kNC = kGainConsumerWarps * 32;

    extern __shared__ __align__(128) unsigned char smem[];
    T* stage_base = reinterpret_cast<T*>(smem);
    T* f_s = reinterpret_cast<T*>(smem + kGainStages * kGainTileBytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kGainStages * kGainTileBytes +
                                                 round_up_int(f_len * (int)sizeof(T), 16));
    uint64_t* empty = full + kGainStages;
    uint64_t* unit_bar = empty + kGainStages;
    double* red = reinterpret_cast<double*>(unit_bar + kRedRing);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(red + kRedRing * kGainConsumerWarps);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // the cells of the binary domain, or every cell when there is no list
    const int cell = cell_list ? cell_list[blockIdx.y] : (int)blockIdx.y;

    if (tid == 0) {
        for (int s = 0; s < kGainStages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), kGainConsumerWarps);
        }
        for (int s = 0; s < kRedRing; ++s) mbar_init(smem_u32(&unit_bar[s]), kGainConsumerWarps);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();  // barriers initialised; the producer may stream G before f is ready

    if (warp == kGainConsumerWarps) {
        // ---------------- producer: one thread issues the bulk copies
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x) {
                const GainUnit U = units[u];
                if (U.tile_b <= 0 || U.n2p <= 0 || U.tile_b * U.n2p > kTileElems) {
                    atomicOr(err, KERR_BAD_UNIT);
                    *abort_flag = 1;
                    ok = false;
                    break;
                }
                const int nt = (U.nb + U.tile_b - 1) / U.tile_b;
                for (int t = 0; t < nt; ++t, ++it) {
                    const int st = it % kGainStages;
                    const uint32_t ph = (it / kGainStages) & 1u;
                    if (!mbar_wait_bounded(smem_u32(&empty[st]), ph ^ 1u, abort_flag)) {
                        if (!*abort_flag) atomicOr(err, KERR_TIMEOUT_EMPTY);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    const int rows = min(U.tile_b, U.nb - t * U.tile_b);
                    const uint32_t bytes = (uint32_t)rows * (uint32_t)U.n2p * (uint32_t)sizeof(T);
                    mbar_arrive_expect_tx(smem_u32(&full[st]), bytes);
                    bulk_g2s(smem_u32(stage_base + (size_t)st * kTileElems),
                             G + U.g_off + (long long)t * U.tile_b * U.n2p, bytes, smem_u32(&full[st]));
                }
            }
            // Wait for this block's own copies before the block may exit.
            const uint32_t first = it > (uint32_t)kGainStages ? it - kGainStages : 0u;
            volatile int never = 0;
            for (uint32_t k = first; k < it; ++k) {
                if (!mbar_wait_bounded(smem_u32(&full[k % kGainStages]), (k / kGainStages) & 1u, &never))
                    atomicOr(err, KERR_TIMEOUT_DRAIN);
            }
        }
        return;
    }

    // ---------------- consumers: 8 warps
    // The work table is static: the block's first unit is read before the wait.
    GainUnit U0{};
    if ((int)blockIdx.x < n_units) U0 = units[blockIdx.x];
    // f is the previous step's output and the previous step still reads the partials this
    // kernel writes: wait for it (the G tiles already stream in meanwhile)
    pdl_wait();
    if (tid == 0) pdl_trigger();
    {
        // f of this cell in the padded per-species layout; zeros in the padding.
        const T* fc = f + (size_t)cell * n_mom;
        for (int i = tid; i < f_len; i += kNC) {
            int s = 0;
            while (s + 1 < so.n && i >= so.offp[s + 1]) ++s;
            const int j = i - so.offp[s];
            const int ns = so.off[s + 1] - so.off[s];
            f_s[i] = (j < ns) ? fc[so.off[s] + j] : T(0);
        }
    }
    asm volatile("bar.sync 1, %0;" ::"n"(kNC) : "memory");  // the consumer warps only
    uint32_t it = 0;
    uint32_t lk = 0;  // units done by this block
    for (int u = blockIdx.x; u < n_units; u += gridDim.x, ++lk) {
        const GainUnit U = u == (int)blockIdx.x ? U0 : units[u];
        if (U.tile_b <= 0 || U.n2p <= 0 || U.tile_b * U.n2p > kTileElems) return;
        const int nt = (U.nb + U.tile_b - 1) / U.tile_b;
        const int nvr = U.n2p / V::n;  // vectors per b-row
        const int dr = kNC / nvr, dcv = kNC - dr * nvr;
        const T* f2 = f_s + U.c_off;
        double acc = 0.0;
        for (int t = 0; t < nt; ++t, ++it) {
            const int st = it % kGainStages;
            const uint32_t ph = (it / kGainStages) & 1u;
            if (!mbar_wait_bounded(smem_u32(&full[st]), ph, abort_flag)) {
                if (!*abort_flag) atomicOr(err, KERR_TIMEOUT_FULL);
                *abort_flag = 1;
                return;
            }
            const int rows = min(U.tile_b, U.nb - t * U.tile_b);
            const vec_t* tile = reinterpret_cast<const vec_t*>(stage_base + (size_t)st * kTileElems);
            const T* f1 = f_s + U.b_off + t * U.tile_b;
            int r = tid / nvr, cv = tid - r * nvr;
            while (r < rows) {
                const vec_t g = tile[r * nvr + cv];
                const vec_t x = reinterpret_cast<const vec_t*>(f2)[cv];
                const T d = V::dot(g, x);
                acc = fma((double)f1[r], (double)d, acc);
                cv += dcv;
                r += dr;
                if (cv >= nvr) {
                    cv -= nvr;
                    ++r;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&empty[st]));
        }
        acc = warp_sum(acc);
        const int slot = lk % kRedRing;
        if (lane == 0) {
            red[slot * kGainConsumerWarps + warp] = acc;
            mbar_arrive(smem_u32(&unit_bar[slot]));
        }
        if (tid == 0) {
            if (!mbar_wait_bounded(smem_u32(&unit_bar[slot]), (lk / kRedRing) & 1u, abort_flag)) {
                if (!*abort_flag) atomicOr(err, KERR_TIMEOUT_FULL);
                *abort_flag = 1;
                return;
            }
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < kGainConsumerWarps; ++w) s += red[slot * kGainConsumerWarps + w];
            partial[(size_t)cell * n_units + u] = s;
        }
    }
}

int gain_stream_blocks_per_sm(int elem_size, int f_smem_len) {
    int n = 0;
    const int smem = gain_stream_smem_bytes(elem_size, f_smem_len);
    if (elem_size == 8) {
        cudaFuncSetAttribute(gain_stream_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, gain_stream_kernel<double>, kGainThreads, smem);
    } else {
        cudaFuncSetAttribute(gain_stream_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, gain_stream_kernel<float>, kGainThreads, smem);
    }
    return n;
}

template <typename T>
cudaError_t launch_gain_stream(const T* G, const GainUnit* units, int n_units, const T* f, int n_mom,
                               const int* sp_off_host, int n_species, int f_smem_len, double* partial,
                               int n_space, int grid_x, int* err, cudaStream_t s, const int* cell_list, bool pdl) {
    // n_space: cells to run (grid y); cell_list maps them to cells, or null for 0..n_space-1
    // sp_off_host: [0..n_species] unpadded then [0..n_species] padded offsets (host array)
    SpOff so;
    so.n = n_species;
    for (int i = 0; i <= n_species; ++i) {
        so.off[i] = sp_off_host[i];
        so.offp[i] = sp_off_host[n_species + 1 + i];
    }
    // the dynamic shared-memory limit was raised by gain_stream_blocks_per_sm at commit
    const int smem = gain_stream_smem_bytes(sizeof(T), f_smem_len);
    dim3 grid(grid_x, n_space);
    // pdl: a step's own sequence (its G is static); a caller's G may be its predecessor's output,
    // which the producer (it starts before the dependency wait) must not read early
    if (pdl)
        return launch_pdl(gain_stream_kernel<T>, grid, dim3(kGainThreads), (size_t)smem, s, G, units, n_units, f, n_mom,
                          so, f_smem_len, partial, err, cell_list);
    gain_stream_kernel<T><<<grid, kGainThreads, smem, s>>>(G, units, n_units, f, n_mom, so, f_smem_len, partial, err,
                                                           cell_list);
    return cudaGetLastError();
}

template cudaError_t launch_gain_stream<double>(const double*, const GainUnit*, int, const double*, int,
                                                const int*, int, int, double*, int, int, int*, cudaStream_t,
                                                const int*, bool);
template cudaError_t launch_gain_stream<float>(const float*, const GainUnit*, int, const float*, int,
                                               const int*, int, int, double*, int, int, int*, cudaStream_t,
                                               const int*, bool);

// ------------------------------------------------------------------ euler_rows
template <typename T>
__global__ void __launch_bounds__(kRowsWarps * 32) euler_rows_kernel(RowOps<T> ops, const T* __restrict__ f_in,
                                                                     T* __restrict__ f_out, double dt_imm,
                                                                     const double* __restrict__ dt_arr,
                                                                     const unsigned long long* ctr, int kpos,
                                                                     int verbose, double* rec) {
    __shared__ double s_red[kRowsWarps][kStepRecFields];
    // The previous step's state and the step counter (which advances only between step
    // sequences) were final before this grid could launch: as a programmatic dependent it
    // follows this step's gain kernel, which lets it launch only after that kernel's own wait for
    // the kernels before it; without a gain kernel it launches in plain stream order. So the
    // flux, emission and loss products, which read only the state and static operands, run
    // before the wait for this step's gain partials (on SMs beside the gain kernel where it
    // leaves room); everything this grid writes is written after the wait.
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long step = *reinterpret_cast<const volatile unsigned long long*>(ctr) + (unsigned)kpos;
    const double dt_scale = dt_arr ? dt_arr[step] : dt_imm;
    const int i = blockIdx.x * kRowsWarps + warp;

    double m_cr = CUDART_INF, m_bin = CUDART_INF, m_emi = CUDART_INF, m_flux = CUDART_INF;
    double s_df = 0.0, s_f = 0.0;
    const int cell = i < ops.n_state ? i / ops.n_mom : 0;
    const int a = i - cell * ops.n_mom;
    const T* fc = f_in + (size_t)cell * ops.n_mom;
    int s = 0;
    double flux = 0.0, emi = 0.0, loss = 0.0, gain = 0.0;
    // binary term of this cell (SteppingMethods.jl:369): outside BinM.Domain it is zero
    const bool bin_here = i < ops.n_state && ops.has_bin && (ops.bin_on == nullptr || ops.bin_on[cell] != 0);
    if (i < ops.n_state) {
        while (s + 1 < ops.n_species && a >= ops.sp_off[s + 1]) ++s;

        // (a) banded flux row: ELL slots of width ell_w, 128-bit loads of 4 slots per lane
        {
            const T* vrow = ops.ell_val + (size_t)i * ops.ell_w;
            const int* crow = ops.ell_col + (size_t)i * ops.ell_w;
            for (int k = lane * 4; k < ops.ell_w; k += 128) {
                const int4 c4 = *reinterpret_cast<const int4*>(crow + k);
                T v0, v1, v2, v3;
                if constexpr (sizeof(T) == 4) {
                    const float4 v4 = *reinterpret_cast<const float4*>(vrow + k);
                    v0 = v4.x; v1 = v4.y; v2 = v4.z; v3 = v4.w;
                } else {
                    const double2 va = *reinterpret_cast<const double2*>(vrow + k);
                    const double2 vb = *reinterpret_cast<const double2*>(vrow + k + 2);
                    v0 = va.x; v1 = va.y; v2 = vb.x; v3 = vb.y;
                }
                // padding slots carry column -1: only stored entries take part, like a CSC product
                if (c4.x >= 0) flux += (double)v0 * (double)f_in[c4.x];
                if (c4.y >= 0) flux += (double)v1 * (double)f_in[c4.y];
                if (c4.z >= 0) flux += (double)v2 * (double)f_in[c4.z];
                if (c4.w >= 0) flux += (double)v3 * (double)f_in[c4.w];
            }
        }
        // (c) emission row pieces
        if (ops.has_emi) {
            for (int p = ops.emi_rptr[i]; p < ops.emi_rptr[i + 1]; ++p) {
                const int pc = ops.emi_piece[p];
                const T* row = ops.emi_data + ops.emi_data_off[pc] + (size_t)(i - ops.emi_row0[pc]) * ops.emi_ld[pc];
                const T* fx = f_in + ops.emi_col0[pc];
                const int nc = ops.emi_ncols[pc];
                for (int c = lane; c < nc; c += 32) emi += (double)row[c] * (double)fx[c];
            }
        }
        // loss bilinear term
        if (bin_here) {
            const int la = a - ops.sp_off[s];
            for (int b = ops.loss_ptr[s]; b < ops.loss_ptr[s + 1]; ++b) {
                const T* row = ops.loss_data + ops.loss_data_off[b] + (size_t)la * ops.loss_ld[b];
                const T* fx = fc + ops.loss_col_off[b];
                const int nc = ops.loss_ncols[b];
                for (int c = lane; c < nc; c += 32) loss += (double)row[c] * (double)fx[c];
            }
        }
        flux = warp_sum(flux);
        emi = warp_sum(emi);
        loss = warp_sum(loss);
    }
    // The row's unit range, old state and vectors are static or the previous step's: read them
    // before the wait too, so only the gain partials' round trip follows it.
    int u_lo = 0, u_hi = 0;
    T fa = T(0), iap = T(0), injv = T(0), volc = T(0);
    if (i < ops.n_state) {
        if (bin_here) {
            u_lo = ops.unit_ptr[a];
            u_hi = ops.unit_ptr[a + 1];
        }
        if (lane == 0) {
            fa = fc[a];
            iap = ops.invAp[i];
            if (ops.mode == 0) injv = ops.inj[i];
            if (bin_here) volc = ops.vol[cell];
        }
    }
    pdl_wait();  // this step's gain partials (and, in the space pass, the momentum pass) are complete
    if (threadIdx.x == 0) pdl_trigger();
    if (i < ops.n_state) {
        if (bin_here) {
            const double* pr = ops.partial + (size_t)cell * ops.n_units;
            for (int u = u_lo + lane; u < u_hi; u += 32) gain += pr[u];
        }
        gain = warp_sum(gain);

        if (lane == 0 && ops.mode == 1) {
            // ForwardSymplecticEuler momentum pass (SteppingMethods.jl:140-160)
            T df = -(T)flux;
            if (ops.has_emi) df = df + (T)emi;
            if (ops.has_bin) df = df + (bin_here ? (T)((double)volc * (gain - (double)fa * loss)) : T(0));
            df = (T)((double)df * ((double)iap * dt_scale));
            T fm = fa + df;
            fm = jl_mul_bool(fm, fm >= (T)ops.thr_mom);
            f_out[i] = fm;
            ops.dfm_out[i] = df;
        }
        if (lane == 0 && ops.mode == 0) {
            const T dflux = (T)flux;
            const T demi = (T)emi;
            const T dbin = bin_here ? (T)((double)volc * (gain - (double)fa * loss)) : T(0);
            // SteppingMethods.jl:31-46
            T df = -dflux;
            if (ops.has_emi) df = df + demi;
            if (ops.has_bin) df = df + dbin;
            df = (T)((double)df * ((double)iap * dt_scale));
            // :97-101, arithmetic in Float64 like Julia's promotion, one rounding at the store
            const double fnew = (double)fa + ((double)df + (double)injv * dt_scale);
            T fn = (T)fnew;
            fn = jl_mul_bool(fn, fn >= (T)ops.thr);
            fn = jl_mul_bool(fn, fn != (T)CUDART_INF);
            f_out[i] = fn;
            // :48-94 diagnostics on the old f
            const double fd = (double)fa;
            m_cr = nan_to_inf((double)df / fd);
            if (verbose == 3) {
                if (ops.has_bin) m_bin = nan_to_inf((double)dbin / fd);
                if (ops.has_emi) m_emi = nan_to_inf((double)demi / fd);
                m_flux = nan_to_inf(-(double)dflux / fd);
            }
            s_df = (double)df;
            s_f = fd;
        }
    }
    if (ops.mode == 1) return;  // the space pass writes the step's records
    // this block's record; the step's records are reduced by step_diag_kernel, so no row
    // block waits for the others
    if (lane == 0) {
        s_red[warp][0] = m_cr;
        s_red[warp][1] = m_bin;
        s_red[warp][2] = m_emi;
        s_red[warp][3] = m_flux;
        s_red[warp][4] = s_df;
        s_red[warp][5] = s_f;
    }
    __syncthreads();
    if (threadIdx.x < kStepRecFields) {
        // one thread per field, the warps in order: fields 0-3 are minima, 4-5 sums
        const int k = threadIdx.x;
        double r = s_red[0][k];
        for (int w = 1; w < kRowsWarps; ++w) r = k < 4 ? jl_min(r, s_red[w][k]) : r + s_red[w][k];
        rec[(size_t)blockIdx.x * kStepRecFields + k] = r;
    }
}

int euler_rows_blocks(int n_state) { return (n_state + kRowsWarps - 1) / kRowsWarps; }

// Block k reduces the row-block records of step *ctr + k with a fixed assignment (record b to
// thread b mod 256, in order) and a fixed tree, so a step's record does not depend on block
// completion order or on how the steps were grouped into launches.
__global__ void __launch_bounds__(kRowsWarps * 32) step_diag_kernel(const double* __restrict__ blk_red,
                                                                    int n_blocks, int n_steps,
                                                                    unsigned long long* ctr, StepDiagDev* hist,
                                                                    long long hist_cap, int verbose,
                                                                    int has_bin, int has_emi, int sympl,
                                                                    unsigned* ticket) {
    __shared__ double s_fin[kStepRecFields][kRowsWarps * 32];
    pdl_wait();  // the last step's row blocks have written their records
    // a gain kernel that follows may start streaming its (static) blocks; it reads the state and
    // the row kernel after it reads the counter only after this grid has finished
    if (threadIdx.x == 0) pdl_trigger();
    const unsigned long long step0 = *reinterpret_cast<volatile unsigned long long*>(ctr);
    const double* recs = blk_red + (size_t)blockIdx.x * n_blocks * kStepRecFields;
    double r[kStepRecFields] = {CUDART_INF, CUDART_INF, CUDART_INF, CUDART_INF, 0.0, 0.0};
    for (int b = threadIdx.x; b < n_blocks; b += blockDim.x) {
        const double* src = recs + (size_t)b * kStepRecFields;
        for (int k = 0; k < 4; ++k) r[k] = jl_min(r[k], __ldcg(src + k));
        r[4] += __ldcg(src + 4);
        r[5] += __ldcg(src + 5);
    }
    for (int k = 0; k < kStepRecFields; ++k) s_fin[k][threadIdx.x] = r[k];
    __syncthreads();
    for (int o = kRowsWarps * 16; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            for (int k = 0; k < 4; ++k) s_fin[k][threadIdx.x] = jl_min(s_fin[k][threadIdx.x], s_fin[k][threadIdx.x + o]);
            s_fin[4][threadIdx.x] += s_fin[4][threadIdx.x + o];
            s_fin[5][threadIdx.x] += s_fin[5][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < kStepRecFields; ++k) r[k] = s_fin[k][0];
        StepDiagDev d;
        const bool on = (verbose == 1 || verbose == 2 || verbose == 3) && r[5] != 0.0;
        d.cr[0] = on ? -r[0] : 0.0;
        d.cr[1] = (on && verbose == 3 && has_bin && !sympl) ? -r[1] : 0.0;
        d.cr[2] = (on && verbose == 3 && has_emi && !sympl) ? -r[2] : 0.0;
        d.cr[3] = (on && verbose == 3 && !sympl) ? -r[3] : 0.0;
        d.sum_df = r[4];
        d.sum_f = r[5];
        // the symplectic method has no finite check (SteppingMethods.jl:120-243)
        d.finite = (sympl || isfinite(r[4])) ? 1 : 0;
        d.pad = 0;
        hist[(step0 + blockIdx.x) % (unsigned long long)hist_cap] = d;
        // every block has read the counter before it takes its ticket; the last one advances it
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        if (t == gridDim.x - 1) {
            *ticket = 0u;
            *reinterpret_cast<volatile unsigned long long*>(ctr) = step0 + (unsigned long long)n_steps;
        }
    }
}

cudaError_t launch_step_diag(const double* blk_red, int n_blocks, int n_steps, unsigned long long* ctr,
                             StepDiagDev* hist, long long hist_cap, int verbose, int has_bin, int has_emi, int sympl,
                             unsigned* ticket, cudaStream_t s) {
    return launch_pdl(step_diag_kernel, dim3(n_steps), dim3(kRowsWarps * 32), 0, s, blk_red, n_blocks, n_steps, ctr,
                      hist, hist_cap, verbose, has_bin, has_emi, sympl, ticket);
}

template <typename T>
cudaError_t launch_euler_rows(const RowOps<T>& ops, const T* f_in, T* f_out, double dt_imm, const double* dt_arr,
                              const unsigned long long* ctr, int kpos, int verbose, double* rec, bool pdl,
                              cudaStream_t s) {
    const int grid = euler_rows_blocks(ops.n_state);
    if (pdl)
        return launch_pdl(euler_rows_kernel<T>, grid, dim3(kRowsWarps * 32), 0, s, ops, f_in, f_out, dt_imm, dt_arr,
                          ctr, kpos, verbose, rec);
    euler_rows_kernel<T><<<grid, kRowsWarps * 32, 0, s>>>(ops, f_in, f_out, dt_imm, dt_arr, ctr, kpos, verbose, rec);
    return cudaGetLastError();
}

template cudaError_t launch_euler_rows<double>(const RowOps<double>&, const double*, double*, double, const double*,
                                               const unsigned long long*, int, int, double*, bool, cudaStream_t);
template cudaError_t launch_euler_rows<float>(const RowOps<float>&, const float*, float*, double, const double*,
                                              const unsigned long long*, int, int, double*, bool, cudaStream_t);

// ------------------------------------------------------------------ sympl_space
// ForwardSymplecticEuler space pass (SteppingMethods.jl:165-237): one warp per row,
// df_Space = -(X f_Momentum) invAp dt/dt0, f_Space = clamp(f_Momentum + df_Space, 1f-20), then
// f = f_Space + inj dt/dt0 clamped with the sign factor of :235 and the Inf fix of :237.
// Each block writes a record of its rows' (df_Space + df_Momentum) ./ f_old minimum and f_old
// sum in euler_rows' layout; step_diag reduces them to Cr = -min(...) (:217-218).
template <typename T>
__global__ void __launch_bounds__(kRowsWarps * 32) sympl_space_kernel(RowOps<T> ops, const T* __restrict__ f_old,
                                                                      const T* __restrict__ fm,
                                                                      const T* __restrict__ dfm, T* __restrict__ f_out,
                                                                      double dt_imm, const double* __restrict__ dt_arr,
                                                                      const unsigned long long* ctr, int kpos,
                                                                      double* rec) {
    __shared__ double s_red[kRowsWarps][2];
    pdl_wait();  // this step's inputs (gain partials, momentum pass)
    if (threadIdx.x == 0) pdl_trigger();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long step = *reinterpret_cast<const volatile unsigned long long*>(ctr) + (unsigned)kpos;
    const double dt_scale = dt_arr ? dt_arr[step] : dt_imm;
    const int i = blockIdx.x * kRowsWarps + warp;
    double m_cr = CUDART_INF, s_f = 0.0;
    if (i < ops.n_state) {
        double xf = 0.0;
        for (int k = lane; k < ops.x_ell_w; k += 32) {
            const int c = ops.x_ell_col[(size_t)i * ops.x_ell_w + k];
            if (c >= 0) xf += (double)ops.x_ell_val[(size_t)i * ops.x_ell_w + k] * (double)fm[c];
        }
        xf = warp_sum(xf);
        if (lane == 0) {
            const T dsp = (T)((double)(-(T)xf * ops.invAp[i]) * dt_scale);
            T fs = fm[i] + dsp;
            fs = jl_mul_bool(fs, fs >= (T)ops.thr_space);
            T v = (T)((double)fs + (double)ops.inj[i] * dt_scale);
            const T sg = isnan(v) ? v : (v > T(0) ? T(1) : (v < T(0) ? T(-1) : v));
            v = jl_mul_bool(v, v >= (T)ops.thr_space) * sg;
            v = jl_mul_bool(v, v != (T)CUDART_INF);
            f_out[i] = v;
            const double fo = (double)f_old[i];
            m_cr = nan_to_inf((double)(dsp + dfm[i]) / fo);
            s_f = fo;
        }
    }
    if (lane == 0) {
        s_red[warp][0] = m_cr;
        s_red[warp][1] = s_f;
    }
    __syncthreads();
    if (threadIdx.x < kStepRecFields) {
        // fields 0 (minimum) and 5 (sum) over the warps in order; no per-term Crs, no df sum
        const int k = threadIdx.x;
        double r = k == 0 ? s_red[0][0] : (k == 5 ? s_red[0][1] : (k == 4 ? 0.0 : CUDART_INF));
        if (k == 0)
            for (int w = 1; w < kRowsWarps; ++w) r = jl_min(r, s_red[w][0]);
        if (k == 5)
            for (int w = 1; w < kRowsWarps; ++w) r += s_red[w][1];
        rec[(size_t)blockIdx.x * kStepRecFields + k] = r;
    }
}

template <typename T>
cudaError_t launch_sympl_space(const RowOps<T>& ops, const T* f_old, const T* fm, const T* dfm, T* f_out,
                               double dt_imm, const double* dt_arr, const unsigned long long* ctr, int kpos,
                               double* rec, cudaStream_t s) {
    const int grid = euler_rows_blocks(ops.n_state);
    return launch_pdl(sympl_space_kernel<T>, grid, dim3(kRowsWarps * 32), 0, s, ops, f_old, fm, dfm, f_out, dt_imm,
                      dt_arr, ctr, kpos, rec);
}
template cudaError_t launch_sympl_space<double>(const RowOps<double>&, const double*, const double*, const double*,
                                                double*, double, const double*, const unsigned long long*, int,
                                                double*, cudaStream_t);
template cudaError_t launch_sympl_space<float>(const RowOps<float>&, const float*, const float*, const float*, float*,
                                               double, const double*, const unsigned long long*, int, double*,
                                               cudaStream_t);

// ------------------------------------------------------------------ bounded-wait self-test
// One block waits on an mbarrier phase that nothing completes, with a limit of limit_ns, and
// reports the timeout through err: the same give-up path every pipeline wait in this library
// takes, exercised without a fault.
__global__ void bounded_wait_selftest_kernel(unsigned long long limit_ns, int* err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long t0 = globaltimer();
        bool done = false;
        while (!done) {
            done = mbar_try_wait(smem_u32(&bar), 0u);
            if (!done && globaltimer() - t0 > limit_ns) break;
        }
        if (!done) atomicOr(err, KERR_TIMEOUT_FULL);
        mbar_arrive(smem_u32(&bar));  // complete the phase so the barrier is left consistent
    }
}

cudaError_t launch_bounded_wait_selftest(unsigned long long limit_ns, int* err, cudaStream_t s) {
    bounded_wait_selftest_kernel<<<1, 32, 0, s>>>(limit_ns, err);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ helpers
template <typename Tin, typename Tout>
__global__ void pad_rows_kernel(const Tin* __restrict__ src, long long rows, int n, Tout* __restrict__ dst, int np) {
    const long long total = rows * (long long)np;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const long long r = k / np;
        const int c = (int)(k - r * np);
        dst[k] = c < n ? (Tout)src[r * n + c] : Tout(0);
    }
}

template <typename Tin, typename Tout>
cudaError_t launch_pad_rows(const Tin* src, long long rows, int n, Tout* dst, int np, cudaStream_t s) {
    pad_rows_kernel<Tin, Tout><<<148 * 8, 256, 0, s>>>(src, rows, n, dst, np);
    return cudaGetLastError();
}
template cudaError_t launch_pad_rows<double, double>(const double*, long long, int, double*, int, cudaStream_t);
template cudaError_t launch_pad_rows<float, float>(const float*, long long, int, float*, int, cudaStream_t);
template cudaError_t launch_pad_rows<double, float>(const double*, long long, int, float*, int, cudaStream_t);
template cudaError_t launch_pad_rows<float, double>(const float*, long long, int, double*, int, cudaStream_t);

// Per (cell, species) FP64 number and energy sums; out = [n_space][n_species][2].
template <typename T>
__global__ void moments_kernel(const T* __restrict__ f, int n_mom, const int* __restrict__ sp_off,
                               const double* __restrict__ w, double* __restrict__ out, int n_species) {
    __shared__ double s_n[256], s_e[256];
    const int s = blockIdx.x, cell = blockIdx.y;
    const int lo = sp_off[s], hi = sp_off[s + 1];
    double a = 0.0, e = 0.0;
    for (int k = lo + threadIdx.x; k < hi; k += blockDim.x) {
        const double v = (double)f[(size_t)cell * n_mom + k];
        a += v;
        e += v * w[k];
    }
    s_n[threadIdx.x] = a;
    s_e[threadIdx.x] = e;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_n[threadIdx.x] += s_n[threadIdx.x + o];
            s_e[threadIdx.x] += s_e[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[((size_t)cell * n_species + s) * 2 + 0] = s_n[0];
        out[((size_t)cell * n_species + s) * 2 + 1] = s_e[0];
    }
}

cudaError_t launch_moments_f64(const double* f, int n_mom, int n_space, const int* sp_off, int n_species,
                               const double* w, double* out, cudaStream_t s) {
    moments_kernel<double><<<dim3(n_species, n_space), 256, 0, s>>>(f, n_mom, sp_off, w, out, n_species);
    return cudaGetLastError();
}
cudaError_t launch_moments_f32(const float* f, int n_mom, int n_space, const int* sp_off, int n_species,
                               const double* w, double* out, cudaStream_t s) {
    moments_kernel<float><<<dim3(n_species, n_space), 256, 0, s>>>(f, n_mom, sp_off, w, out, n_species);
    return cudaGetLastError();
}

}  // namespace dtb
