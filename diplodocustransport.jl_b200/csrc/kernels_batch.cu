// Kernels of the batched mixed-precision Euler step.
//
// gain_gemm<BN>: the gain contraction of many instances as a GEMM on the 5th-generation
// tensor cores. A = G rows (BF16 hi and lo halves, K-major, 128-byte swizzle) staged by TMA;
// B = X = f1 (x) f2 for BN instances, formed on the fly by producer warps in shared memory as
// BF16 hi and lo halves in the same swizzled K-major layout; D (FP32) lives in tensor memory.
// Per 16-wide K step three MMAs accumulate hi*hi + hi*lo + lo*hi. One elected thread issues
// the MMAs and commits them to mbarriers; every wait is bounded.
//
// mixed_rows: one (32 rows x 32 instances) tile per block: loss and emission (operands stored
// as BF16 hi+lo with per-row scales) as tensor-core tile products, split-K partial sums of the
// gain, banded flux, then the update of SteppingMethods.jl:46-101 with an FP64 compensated
// (Kahan) accumulation of f.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <algorithm>
#include <utility>

#include "batch_internal.h"
#include "pdl.cuh"
#include "umma.cuh"

namespace dtb {

namespace {


template <int BN>
struct GemmCfg {
    static constexpr int NPW = BN / 32 < 4 ? 4 : BN / 32;  // producer / epilogue warps
    static constexpr int THREADS = (NPW + 2) * 32;
    // threads forming one X row, each KW of its 64 K columns: with BN = 64 all four producer
    // warps form X (the X tile is on the critical path of an HBM-bound group: a G stage stays
    // held until the MMAs that read it complete, and they wait for X)
    static constexpr int KS = NPW * 32 / BN;
    static constexpr int KW = kMmaK / KS;
    static constexpr int A_BYTES = kMmaM * 128;             // one half (hi or lo) of an A stage
    static constexpr int B_BYTES = BN * 128;                // one half of a B stage
    // BN = 64: a 4-stage G ring and a 6-stage X ring, so the producers run ahead of the MMAs
    static constexpr int SB = BN == 64 ? 6 : 2;
    static constexpr int SA = BN == 256 ? 3 : 4;
    static constexpr int DATA = SA * 2 * A_BYTES + SB * 2 * B_BYTES;
    static constexpr int BARS = (2 * SA + 2 * SB + 3) * 8;
    static constexpr int SMEM = 1024 + DATA + BARS + 16;   // 1024: alignment slack
    // tensor memory: all 512 columns as 512 / BN accumulators of BN columns; the hi*hi products
    // go round-robin by K tile into the first NHH of them and the hi*lo + lo*hi products into the
    // last, so no FP32 accumulator sums more than a fraction of the split's K range
    static constexpr int NACC = 512 / BN;
    static constexpr int NHH = NACC - 1;
    static_assert(KS >= 1 && KS * BN == NPW * 32 && KW % 8 == 0, "producer threads cover whole 16-byte chunks");
    static_assert(SMEM <= 232448, "gain GEMM shared memory");
};

template <int BN>
__global__ void __launch_bounds__(GemmCfg<BN>::THREADS, 1)
    gain_gemm_kernel(GemmArgs a) {
    using C = GemmCfg<BN>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* a_base = smem;                                // [SA][hi, lo][128 rows x 128 B]
    unsigned char* b_base = smem + C::SA * 2 * C::A_BYTES;       // [SB][hi, lo][BN rows x 128 B]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + C::DATA);
    uint64_t* full_a = bars;
    uint64_t* empty_a = full_a + C::SA;
    uint64_t* full_b = empty_a + C::SA;
    uint64_t* empty_b = full_b + C::SB;
    uint64_t* acc_bar = empty_b + C::SB;
    uint64_t* drain_bar = acc_bar + 1;
    uint64_t* x0_bar = drain_bar + 1;  // the first X tile is written (its state loads are done)
    uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(x0_bar + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int task = blockIdx.x;
    const int n_tile = task % a.n_tiles;
    const int m_tile = (task / a.n_tiles) % a.m_tiles;
    const int split = task / (a.n_tiles * a.m_tiles);
    const int T = a.n_cb * a.N1;
    // K range of this split: within one input-2 block when the splits are aligned to them (the
    // producers then load that block's f2 once), else an even cut of all K tiles
    int t0, t1;
    if (a.splits_per_cb > 0) {
        const int cb = split / a.splits_per_cb, piece = split - cb * a.splits_per_cb;
        t0 = cb * a.N1 + (int)((long long)piece * a.N1 / a.splits_per_cb);
        t1 = cb * a.N1 + (int)((long long)(piece + 1) * a.N1 / a.splits_per_cb);
    } else {
        t0 = split * a.tiles_per_split;
        t1 = min(T, t0 + a.tiles_per_split);
    }
    const int m0 = m_tile * kMmaM, n0 = n_tile * BN;
    // columns of this tile that belong to slots still stepping, rounded up to the MMA's N granule
    const int hi_cols = a.n_space > 1 ? a.n_space * a.Bst : *reinterpret_cast<const volatile int*>(a.active_hi);
    const int n_eff = max(0, min(BN, (hi_cols - n0 + 15) / 16 * 16));
    const int nt = (n_eff > 0 && t1 > t0) ? t1 - t0 : 0;

    if (tid == 0) {
        for (int s = 0; s < C::SA; ++s) {
            mb_init(smem_addr(&full_a[s]), 1);
            mb_init(smem_addr(&empty_a[s]), 1);
        }
        for (int s = 0; s < C::SB; ++s) {
            mb_init(smem_addr(&full_b[s]), BN / 32 * C::KS);  // one arrive per producing warp
            mb_init(smem_addr(&empty_b[s]), 1);
        }
        mb_init(smem_addr(acc_bar), 1);
        mb_init(smem_addr(drain_bar), 1);
        mb_init(smem_addr(x0_bar), BN / 32 * C::KS);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == C::NPW + 1) {  // TMEM: NACC accumulators of BN fp32 columns x 128 lanes
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_holder)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_holder;

    if (warp == C::NPW) {
        // ---------------- bulk-copy producer of the G tiles: the (m tile, K tile) pair is one
        // contiguous, pre-swizzled 32 KB block (hi then lo), streamed in order
        if (lane == 0 && nt > 0) {
            const unsigned char* src0 = a.gt + ((size_t)m_tile * T + t0) * kGTileBytes;
            int j = 0;
            for (; j < nt; ++j) {
                const int sa = j % C::SA;
                const uint32_t ph = (j / C::SA) & 1u;
                if (!mb_wait(smem_addr(&empty_a[sa]), ph ^ 1u, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_EMPTY);
                    *abort_flag = 1;
                    break;
                }
                mb_expect_tx(smem_addr(&full_a[sa]), 2 * C::A_BYTES);
                const unsigned char* src = src0 + (size_t)j * kGTileBytes;
                bulk_load_stream(smem_addr(a_base + (size_t)(sa * 2) * C::A_BYTES), src, C::A_BYTES, smem_addr(&full_a[sa]));
                bulk_load_stream(smem_addr(a_base + (size_t)(sa * 2 + 1) * C::A_BYTES), src + C::A_BYTES, C::A_BYTES,
                          smem_addr(&full_a[sa]));
                // the producers' state loads come first: the rest of the G ring waits for the first
                // X tile, so those loads do not queue behind every CTA's full ring of G traffic
                if (j == 0 && nt > 1 && a.ring_after_x0 && !mb_wait(smem_addr(x0_bar), 0u, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_FULL);
                    *abort_flag = 1;
                    ++j;
                    break;
                }
            }
            // drain: this block's own copies must land before it may exit
            for (int k = j > C::SA ? j - C::SA : 0; k < j; ++k) {
                if (!mb_wait(smem_addr(&full_a[k % C::SA]), (k / C::SA) & 1u, nullptr)) atomicOr(a.err, KERR_TIMEOUT_DRAIN);
            }
        }
    } else if (warp == C::NPW + 1) {
        // ---------------- MMA issuer
        if (lane == 0 && nt > 0) {
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n_eff >> 3) << 17) |
                                   ((uint32_t)(kMmaM >> 4) << 24);
            int issued = 0;
            for (int j = 0; j < nt; ++j) {
                const int sa = j % C::SA, sb = j % C::SB;
                if (!mb_wait(smem_addr(&full_a[sa]), (j / C::SA) & 1u, abort_flag) ||
                    !mb_wait(smem_addr(&full_b[sb]), (j / C::SB) & 1u, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_FULL);
                    *abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t ahi = smem_addr(a_base + (size_t)(sa * 2) * C::A_BYTES);
                const uint32_t alo = smem_addr(a_base + (size_t)(sa * 2 + 1) * C::A_BYTES);
                const uint32_t bhi = smem_addr(b_base + (size_t)(sb * 2) * C::B_BYTES);
                const uint32_t blo = smem_addr(b_base + (size_t)(sb * 2 + 1) * C::B_BYTES);
                const uint64_t dahi = umma_desc_sw128(ahi), dalo = umma_desc_sw128(alo);
                const uint64_t dbhi = umma_desc_sw128(bhi), dblo = umma_desc_sw128(blo);
                const uint32_t d_hh = tmem + (uint32_t)(BN * (j % C::NHH));
                const uint32_t d_lo = tmem + (uint32_t)(BN * C::NHH);
#pragma unroll
                for (int kk = 0; kk < kMmaK / 16; ++kk) {
                    const uint64_t o = (uint64_t)(kk * 2);  // 16 BF16 = 32 bytes = 2 x 16 B
                    umma_bf16(d_hh, dahi + o, dbhi + o, idesc, (j >= C::NHH || kk > 0) ? 1u : 0u);
                    umma_bf16(d_lo, dahi + o, dblo + o, idesc, (j > 0 || kk > 0) ? 1u : 0u);
                    umma_bf16(d_lo, dalo + o, dbhi + o, idesc, 1u);
                }
                umma_commit(smem_addr(&empty_a[sa]));
                umma_commit(smem_addr(&empty_b[sb]));
                ++issued;
            }
            if (*abort_flag) {
                if (issued > 0) {  // let the MMAs already issued finish before tensor memory is freed
                    umma_commit(smem_addr(drain_bar));
                    if (!mb_wait(smem_addr(drain_bar), 0u, nullptr)) atomicOr(a.err, KERR_TIMEOUT_DRAIN);
                }
            } else {
                umma_commit(smem_addr(acc_bar));
            }
        }
    } else {
        // ---------------- X producers (KS threads per instance row, KW of its K columns each),
        // then the epilogue
        const int p = tid % BN;   // row of the B tile
        const int kh = tid / BN;  // K part of the row
        pdl_wait();  // F is the previous step's output
        if (tid == 0) pdl_trigger();
        if (kh < C::KS && nt > 0) {
            // column n0 + p: cell (n0 + p) / Bst of slot (n0 + p) % Bst; the cell's states start at
            // row cell * n_mom of F
            const int col = n0 + p;
            const int cell = col / a.Bst;
            const int inst = col - cell * a.Bst;
            const bool valid = cell < a.n_space && inst < a.Bcap && p < n_eff;
            const float* Fc = a.F + (size_t)(valid ? cell : 0) * a.n_mom * a.Bst;
            const float s1 = valid ? a.isig1[inst] : 0.f;
            const float s2 = valid ? a.isig2[inst] : 0.f;
            float f2r[C::KW];
            int cur_cb = -1;
            // f1[b] of the next tile is loaded one tile ahead so its latency hides behind the
            // current tile's conversion
            float x1_next = 0.f;
            if (valid) {
                const int b0 = t0 - (t0 / a.N1) * a.N1;
                x1_next = __ldg(Fc + (size_t)(a.off1 + b0) * a.Bst + inst);
            }
            for (int j = 0; j < nt; ++j) {
                const int t = t0 + j, cb = t / a.N1;
                const int sb = j % C::SB;
                const float x1 = (x1_next * s1) * s2;  // both scales are powers of two: exact
                if (valid && j + 1 < nt) {
                    const int tn = t + 1, bn = tn - (tn / a.N1) * a.N1;
                    x1_next = __ldg(Fc + (size_t)(a.off1 + bn) * a.Bst + inst);
                }
                if (!mb_wait(smem_addr(&empty_b[sb]), ((j / C::SB) & 1u) ^ 1u, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_EMPTY);
                    *abort_flag = 1;
                    break;
                }
                if (cb != cur_cb) {
                    // KW unconditional loads (clamped in bounds) issued back to back, the padding
                    // zeroed afterwards: one round trip instead of a load-use chain
                    const float* fb = Fc + (valid ? inst : 0);
                    const int cbase = cb * kMmaK + kh * C::KW;
#pragma unroll
                    for (int c = 0; c < C::KW; ++c) {
                        const int cc = min(cbase + c, a.n2 - 1);
                        f2r[c] = __ldg(fb + (size_t)(a.off2 + cc) * a.Bst);
                    }
#pragma unroll
                    for (int c = 0; c < C::KW; ++c)
                        if (!valid || cbase + c >= a.n2) f2r[c] = 0.f;
                    cur_cb = cb;
                }
                unsigned char* rhi = b_base + (size_t)(sb * 2) * C::B_BYTES + (size_t)p * 128;
                unsigned char* rlo = b_base + (size_t)(sb * 2 + 1) * C::B_BYTES + (size_t)p * 128;
#pragma unroll
                for (int q = 0; q < C::KW / 8; ++q) {
                    uint32_t h[4], l[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float v0 = x1 * f2r[8 * q + 2 * e];
                        const float v1 = x1 * f2r[8 * q + 2 * e + 1];
                        const __nv_bfloat162 hh = __floats2bfloat162_rn(v0, v1);
                        const float2 hf = __bfloat1622float2(hh);
                        h[e] = *reinterpret_cast<const uint32_t*>(&hh);
                        l[e] = pack_bf16x2(v0 - hf.x, v1 - hf.y);
                    }
                    // 16-byte chunk kh * KW / 8 + q of the row, at its 128-byte-swizzled place
                    const int phys = (((kh * (C::KW / 8) + q) ^ (p & 7)) << 4);
                    *reinterpret_cast<uint4*>(rhi + phys) = make_uint4(h[0], h[1], h[2], h[3]);
                    *reinterpret_cast<uint4*>(rlo + phys) = make_uint4(l[0], l[1], l[2], l[3]);
                }
                // make this thread's generic-proxy stores visible to the tensor core, then one
                // arrive per warp once every lane has fenced
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    mb_arrive(smem_addr(&full_b[sb]));
                    if (j == 0) mb_arrive(smem_addr(x0_bar));
                }
            }
        }
        // epilogue: TMEM lanes 32*(warp%4).. hold rows m0 + 32*(warp%4) + lane
        const int lg = warp & 3;
        const int ncol = BN / (C::NPW / 4);
        const int c0 = (warp >> 2) * ncol;
        const int row = m0 + lg * 32 + lane;
        bool ok = true;
        if (nt > 0) {
            ok = mb_wait(smem_addr(acc_bar), 0u, abort_flag);
            if (!ok && !*abort_flag) atomicOr(a.err, KERR_TIMEOUT_FULL);
            tc_fence_after();
        }
        if (ok && !*abort_flag) {
            float* dst = a.partial + (size_t)split * a.Bpad * a.M;
            // the hi*hi accumulators that received products (tile j went to j % NHH), then the
            // lo accumulator, summed in that fixed order in FP32 with round-to-nearest; all loads
            // of a 16-column chunk in flight before one wait
            const int n_hh = min(C::NHH, nt);
            for (int cc = 0; cc < ncol; cc += 16) {
                uint32_t r[C::NACC][16];
                const bool live = nt > 0 && c0 + cc < n_eff;
                const uint32_t ta = tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)(c0 + cc);
                if (live) {
#pragma unroll
                    for (int h = 0; h < C::NACC; ++h)
                        if (h < n_hh || h == C::NHH) tmem_ld16_issue(ta + (uint32_t)(BN * h), r[h]);
                    tmem_ld_wait();
                }
                if (row < a.M) {
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        float v = 0.f;
                        if (live) {
                            v = __uint_as_float(r[0][k]);
#pragma unroll
                            for (int h = 1; h < C::NHH; ++h)
                                if (h < n_hh) v += __uint_as_float(r[h][k]);
                            v += __uint_as_float(r[C::NHH][k]);
                        }
                        dst[(size_t)(n0 + c0 + cc + k) * a.M + row] = v;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == C::NPW + 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// ------------------------------------------------------------------ CTA-pair gain GEMM
// The same contraction with the MMA spread over the two SMs of a cluster pair
// (tcgen05.mma.cta_group::2, M = 256 = two m tiles, N = 256 columns of X): each CTA stages its
// own 128 G rows and HALF of the X tile, and the pair's tensor cores read both halves, so an SM
// forms 128 instead of 256 columns of X and its shared memory serves A plus half of B per MMA
// (104 instead of 157 bytes per clock at the full MMA rate, against the 128 an SM delivers).
// The even CTA (rank 0) issues the MMAs for the pair. The odd CTA's producer warps arrive on the
// even CTA's X barrier directly and one odd-CTA thread forwards the landing of each of its G
// stages; the even CTA commits stage releases and the final accumulator to the barriers of
// both. Each CTA copies only its own tiles, from this GPU's memory, into its own shared memory.
struct PairCfg {
    static constexpr int BN = 256;               // X columns of a pair (the MMA's N)
    static constexpr int HN = BN / 2;            // X columns staged by each CTA
    static constexpr int NPW = 8;                // producer / epilogue warps
    static constexpr int THREADS = (NPW + 2) * 32;
    static constexpr int A_BYTES = kMmaM * 128;  // hi or lo of this CTA's 128 G rows x 64 K
    static constexpr int B_BYTES = HN * 128;     // hi or lo of this CTA's half of the X tile
    static constexpr int SA = 4;
    static constexpr int SB = 3;
    static constexpr int DATA = SA * 2 * A_BYTES + SB * 2 * B_BYTES;
    static constexpr int BARS = (3 * SA + 2 * SB + 3) * 8;
    static constexpr int SMEM = 1024 + DATA + BARS + 16;
};
static_assert(PairCfg::SMEM <= 232448, "pair GEMM shared memory");


__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PairCfg::THREADS, 1)
    gain_gemm_pair_kernel(GemmArgs a) {
    using C = PairCfg;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* a_base = smem;                           // [SA][hi, lo][128 rows x 128 B]
    unsigned char* b_base = smem + C::SA * 2 * C::A_BYTES;  // [SB][hi, lo][HN rows x 128 B]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + C::DATA);
    uint64_t* full_a = bars;             // this CTA's G stage landed
    uint64_t* empty_a = full_a + C::SA;  // the pair's MMAs are done with the stage
    uint64_t* pfull_a = empty_a + C::SA; // rank 0 only: the odd CTA's G stage landed
    uint64_t* full_b = pfull_a + C::SA;  // rank 0: both CTAs' X halves of the stage are written
    uint64_t* empty_b = full_b + C::SB;
    uint64_t* acc_bar = empty_b + C::SB;
    uint64_t* drain_bar = acc_bar + 1;
    uint64_t* x0_bar = drain_bar + 1;
    uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(x0_bar + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_rank();
    const int pair = blockIdx.x >> 1;
    const int m_pairs = a.m_tiles >> 1;
    const int n_tile = pair % a.n_tiles;
    const int mp = (pair / a.n_tiles) % m_pairs;
    const int split = pair / (a.n_tiles * m_pairs);
    const int m_tile = 2 * mp + (int)rank;
    const int T = a.n_cb * a.N1;
    int t0, t1;
    if (a.splits_per_cb > 0) {
        const int cb = split / a.splits_per_cb, piece = split - cb * a.splits_per_cb;
        t0 = cb * a.N1 + (int)((long long)piece * a.N1 / a.splits_per_cb);
        t1 = cb * a.N1 + (int)((long long)(piece + 1) * a.N1 / a.splits_per_cb);
    } else {
        t0 = split * a.tiles_per_split;
        t1 = min(T, t0 + a.tiles_per_split);
    }
    const int m0 = m_tile * kMmaM, n0 = n_tile * C::BN;
    // active columns rounded up to 32, so each CTA's half is a whole number of 16-row groups
    const int hi_cols = a.n_space > 1 ? a.n_space * a.Bst : *reinterpret_cast<const volatile int*>(a.active_hi);
    const int n_eff = max(0, min(C::BN, (hi_cols - n0 + 31) / 32 * 32));
    const int hn = n_eff / 2;
    const int nt = (n_eff > 0 && t1 > t0) ? t1 - t0 : 0;
    // X producers (warps 0 .. NPW-1): row c of this CTA's half (column n0 + rank * hn + c), two
    // threads per row, each converting one 32-wide half of the 64-wide K tile. Their wait for the
    // previous step and their first state loads overlap the pair's set-up: they arrive on the
    // cluster barrier first and wait on it after the loads.
    const bool producer = warp < C::NPW;
    const int c = tid & (C::HN - 1), kh = tid / C::HN;
    bool valid = false;
    const float* Fc = a.F;
    float s1 = 0.f, s2 = 0.f, x1_next = 0.f;
    int inst = 0, cur_cb = -1;
    float f2r[kMmaK / 2];

    if (tid == 0) {
        for (int s = 0; s < C::SA; ++s) {
            mb_init(smem_addr(&full_a[s]), 1);
            mb_init(smem_addr(&empty_a[s]), 1);
            mb_init(smem_addr(&pfull_a[s]), 1);
        }
        for (int s = 0; s < C::SB; ++s) {
            mb_init(smem_addr(&full_b[s]), 2 * C::NPW);  // one arrive per producing warp of the pair
            mb_init(smem_addr(&empty_b[s]), 1);
        }
        mb_init(smem_addr(acc_bar), 1);
        mb_init(smem_addr(drain_bar), 1);
        mb_init(smem_addr(x0_bar), C::NPW);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == C::NPW + 1) {  // same warp in both CTAs: two accumulators of BN fp32 columns x 128 lanes
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_holder)),
                     "r"(2 * C::BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    // both CTAs' barriers are initialised before either CTA signals the other
    tc_fence_before();
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    if (producer) {
        pdl_wait();  // F is the previous step's output, and the previous epilogue reads the partials
        if (tid == 0) pdl_trigger();
        if (nt > 0) {
            const int col = n0 + (int)rank * hn + c;
            const int cell = col / a.Bst;
            inst = col - cell * a.Bst;
            valid = c < hn && cell < a.n_space && inst < a.Bcap;
            Fc = a.F + (size_t)(valid ? cell : 0) * a.n_mom * a.Bst;
            s1 = valid ? a.isig1[inst] : 0.f;
            s2 = valid ? a.isig2[inst] : 0.f;
            if (valid) {
                const int b0 = t0 - (t0 / a.N1) * a.N1;
                x1_next = __ldg(Fc + (size_t)(a.off1 + b0) * a.Bst + inst);
            }
            // the first tile's 32 input-2 values (clamped in bounds, padding zeroed after)
            const int cb0 = t0 / a.N1;
            const float* fb = Fc + (valid ? inst : 0);
            const int cbase = cb0 * kMmaK + kh * (kMmaK / 2);
#pragma unroll
            for (int e = 0; e < kMmaK / 2; ++e) {
                const int cc = min(cbase + e, a.n2 - 1);
                f2r[e] = __ldg(fb + (size_t)(a.off2 + cc) * a.Bst);
            }
#pragma unroll
            for (int e = 0; e < kMmaK / 2; ++e)
                if (!valid || cbase + e >= a.n2) f2r[e] = 0.f;
            cur_cb = cb0;
        }
    }
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    tc_fence_after();
    const uint32_t tmem = *tmem_holder;

    if (warp == C::NPW) {
        // ---------------- bulk-copy producer of this CTA's G tiles
        if (lane == 0 && nt > 0) {
            const unsigned char* src0 = a.gt + ((size_t)m_tile * T + t0) * kGTileBytes;
            int j = 0;
            for (; j < nt; ++j) {
                const int sa = j % C::SA;
                const uint32_t ph = (j / C::SA) & 1u;
                if (!mb_wait(smem_addr(&empty_a[sa]), ph ^ 1u, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_EMPTY);
                    *abort_flag = 1;
                    break;
                }
                mb_expect_tx(smem_addr(&full_a[sa]), 2 * C::A_BYTES);
                const unsigned char* src = src0 + (size_t)j * kGTileBytes;
                bulk_load_stream(smem_addr(a_base + (size_t)(sa * 2) * C::A_BYTES), src, C::A_BYTES, smem_addr(&full_a[sa]));
                bulk_load_stream(smem_addr(a_base + (size_t)(sa * 2 + 1) * C::A_BYTES), src + C::A_BYTES, C::A_BYTES,
                          smem_addr(&full_a[sa]));
                // the first two G tiles go out at once, the rest after the first X tile (so the
                // producers' state loads do not queue behind the whole ring of G traffic)
                if (j == 1 && nt > 2 && a.ring_after_x0 && !mb_wait(smem_addr(x0_bar), 0u, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_FULL);
                    *abort_flag = 1;
                    ++j;
                    break;
                }
            }
            for (int k = j > C::SA ? j - C::SA : 0; k < j; ++k) {
                if (!mb_wait(smem_addr(&full_a[k % C::SA]), (k / C::SA) & 1u, nullptr)) atomicOr(a.err, KERR_TIMEOUT_DRAIN);
            }
        }
    } else if (warp == C::NPW + 1) {
        if (lane == 0 && nt > 0 && rank == 0) {
            // ---------------- MMA issuer of the pair
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n_eff >> 3) << 17) |
                                   ((uint32_t)((2 * kMmaM) >> 4) << 24);
            int issued = 0;
            for (int j = 0; j < nt; ++j) {
                const int sa = j % C::SA, sb = j % C::SB;
                const uint32_t pa = (j / C::SA) & 1u, pb = (j / C::SB) & 1u;
                if (!mb_wait(smem_addr(&full_a[sa]), pa, abort_flag) ||
                    !mb_wait(smem_addr(&pfull_a[sa]), pa, abort_flag) ||
                    !mb_wait(smem_addr(&full_b[sb]), pb, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_FULL);
                    *abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t ahi = smem_addr(a_base + (size_t)(sa * 2) * C::A_BYTES);
                const uint32_t alo = smem_addr(a_base + (size_t)(sa * 2 + 1) * C::A_BYTES);
                const uint32_t bhi = smem_addr(b_base + (size_t)(sb * 2) * C::B_BYTES);
                const uint32_t blo = smem_addr(b_base + (size_t)(sb * 2 + 1) * C::B_BYTES);
                const uint64_t dahi = umma_desc_sw128(ahi), dalo = umma_desc_sw128(alo);
                const uint64_t dbhi = umma_desc_sw128(bhi), dblo = umma_desc_sw128(blo);
                // hi*hi into the first accumulator, hi*lo + lo*hi into the second
#pragma unroll
                for (int kk = 0; kk < kMmaK / 16; ++kk) {
                    const uint64_t o = (uint64_t)(kk * 2);
                    umma2_bf16(tmem, dahi + o, dbhi + o, idesc, (j > 0 || kk > 0) ? 1u : 0u);
                    umma2_bf16(tmem + C::BN, dahi + o, dblo + o, idesc, (j > 0 || kk > 0) ? 1u : 0u);
                    umma2_bf16(tmem + C::BN, dalo + o, dbhi + o, idesc, 1u);
                }
                umma2_commit(smem_addr(&empty_a[sa]));
                umma2_commit(peer_addr(smem_addr(&empty_a[sa]), 1u));
                umma2_commit(smem_addr(&empty_b[sb]));
                umma2_commit(peer_addr(smem_addr(&empty_b[sb]), 1u));
                ++issued;
            }
            if (*abort_flag) {
                if (issued > 0) {  // the MMAs already issued read both CTAs' shared memory
                    umma2_commit(smem_addr(drain_bar));
                    if (!mb_wait(smem_addr(drain_bar), 0u, nullptr)) atomicOr(a.err, KERR_TIMEOUT_DRAIN);
                }
            } else {
                umma2_commit(smem_addr(acc_bar));
                umma2_commit(peer_addr(smem_addr(acc_bar), 1u));
            }
        } else if (lane == 0 && nt > 0) {
            // ---------------- odd CTA: forward each landed G stage to the even CTA, in order
            for (int j = 0; j < nt; ++j) {
                const int sa = j % C::SA;
                if (!mb_wait(smem_addr(&full_a[sa]), (j / C::SA) & 1u, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_FULL);
                    *abort_flag = 1;
                    break;
                }
                mb_arrive_remote(peer_addr(smem_addr(&pfull_a[sa]), 0u));
            }
        }
    } else {
        // ---------------- X producers (their first state loads were issued during the set-up)
        if (nt > 0) {
            for (int j = 0; j < nt; ++j) {
                const int t = t0 + j, cb = t / a.N1;
                const int sb = j % C::SB;
                const float x1 = (x1_next * s1) * s2;  // both scales are powers of two: exact
                if (valid && j + 1 < nt) {
                    const int tn = t + 1, bn = tn - (tn / a.N1) * a.N1;
                    x1_next = __ldg(Fc + (size_t)(a.off1 + bn) * a.Bst + inst);
                }
                if (!mb_wait(smem_addr(&empty_b[sb]), ((j / C::SB) & 1u) ^ 1u, abort_flag)) {
                    if (!*abort_flag) atomicOr(a.err, KERR_TIMEOUT_EMPTY);
                    *abort_flag = 1;
                    break;
                }
                if (cb != cur_cb) {
                    const float* fb = Fc + (valid ? inst : 0);
                    const int cbase = cb * kMmaK + kh * (kMmaK / 2);
#pragma unroll
                    for (int e = 0; e < kMmaK / 2; ++e) {
                        const int cc = min(cbase + e, a.n2 - 1);
                        f2r[e] = __ldg(fb + (size_t)(a.off2 + cc) * a.Bst);
                    }
#pragma unroll
                    for (int e = 0; e < kMmaK / 2; ++e)
                        if (!valid || cbase + e >= a.n2) f2r[e] = 0.f;
                    cur_cb = cb;
                }
                unsigned char* rhi = b_base + (size_t)(sb * 2) * C::B_BYTES + (size_t)c * 128;
                unsigned char* rlo = b_base + (size_t)(sb * 2 + 1) * C::B_BYTES + (size_t)c * 128;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint32_t h[4], l[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float v0 = x1 * f2r[8 * q + 2 * e];
                        const float v1 = x1 * f2r[8 * q + 2 * e + 1];
                        const __nv_bfloat162 hh = __floats2bfloat162_rn(v0, v1);
                        const float2 hf = __bfloat1622float2(hh);
                        h[e] = *reinterpret_cast<const uint32_t*>(&hh);
                        l[e] = pack_bf16x2(v0 - hf.x, v1 - hf.y);
                    }
                    const int phys = (((kh * 4 + q) ^ (c & 7)) << 4);
                    *reinterpret_cast<uint4*>(rhi + phys) = make_uint4(h[0], h[1], h[2], h[3]);
                    *reinterpret_cast<uint4*>(rlo + phys) = make_uint4(l[0], l[1], l[2], l[3]);
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    if (rank == 0)
                        mb_arrive(smem_addr(&full_b[sb]));
                    else
                        mb_arrive_remote(peer_addr(smem_addr(&full_b[sb]), 0u));
                    if (j == 0) mb_arrive(smem_addr(x0_bar));
                }
            }
        }
        // epilogue: this CTA's TMEM holds its 128 G rows x the pair's n_eff columns
        const int lg = warp & 3;
        const int ncol = C::BN / (C::NPW / 4);
        const int c0 = (warp >> 2) * ncol;
        const int row = m0 + lg * 32 + lane;
        bool ok = true;
        if (nt > 0) {
            ok = mb_wait(smem_addr(acc_bar), 0u, abort_flag);
            if (!ok && !*abort_flag) atomicOr(a.err, KERR_TIMEOUT_FULL);
            tc_fence_after();
        }
        if (ok && !*abort_flag) {
            // the warp's 128 columns, 64 at a time: both accumulators' loads in flight before one
            // wait, then hi*hi + (hi*lo + lo*hi) in FP32 with round-to-nearest
            static_assert(C::BN / (C::NPW / 4) == 128, "epilogue covers 128 columns per warp");
            float* dst = a.partial + (size_t)split * a.Bpad * a.M + (size_t)(n0 + c0) * a.M + row;
            const uint32_t ta = tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)c0;
#pragma unroll
            for (int hf = 0; hf < 2; ++hf) {
                uint32_t rv[4][16], rl[4][16];
                if (nt > 0 && c0 + 64 * hf < n_eff) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        tmem_ld16_issue(ta + 64 * hf + 16 * q, rv[q]);
                        tmem_ld16_issue(ta + C::BN + 64 * hf + 16 * q, rl[q]);
                    }
                    tmem_ld_wait();
                }
                if (row < a.M) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const bool live = nt > 0 && c0 + 64 * hf + 16 * q < n_eff;
#pragma unroll
                        for (int k = 0; k < 16; ++k)
                            dst[(size_t)(64 * hf + 16 * q + k) * a.M] =
                                live ? __uint_as_float(rv[q][k]) + __uint_as_float(rl[q][k]) : 0.f;
                    }
                }
            }
        }
    }
    // neither CTA leaves (or frees tensor memory) while the other may still touch its shared
    // memory, barriers or tensor memory
    __syncwarp();
    tc_fence_before();
    cluster_sync_all();
    if (warp == C::NPW + 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * C::BN) : "memory");
    }
}

}  // namespace

int gain_gemm_smem_bytes(int bn) {
    switch (bn) {
        case 64: return GemmCfg<64>::SMEM;
        case 128: return GemmCfg<128>::SMEM;
        default: return GemmCfg<256>::SMEM;
    }
}

cudaError_t prepare_gain_gemm(int bn) {
    switch (bn) {
        case 64:
            return cudaFuncSetAttribute(gain_gemm_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmCfg<64>::SMEM);
        case 128:
            return cudaFuncSetAttribute(gain_gemm_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        GemmCfg<128>::SMEM);
        case 256:
            return cudaFuncSetAttribute(gain_gemm_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        GemmCfg<256>::SMEM);
        default:
            return cudaErrorInvalidValue;
    }
}

// The dynamic shared-memory limit is raised once per device by prepare_gain_gemm (commit time),
// so launches stay legal inside a stream capture.
template <int BN>
static cudaError_t launch_gemm_bn(const GemmArgs& a, cudaStream_t s) {
    using C = GemmCfg<BN>;
    const int grid = a.m_tiles * a.n_tiles * a.n_splits;
    return launch_pdl(gain_gemm_kernel<BN>, dim3(grid), dim3(C::THREADS), C::SMEM, s, a);
}

cudaError_t prepare_gain_gemm_pair(int* max_pairs) {
    cudaError_t e = cudaFuncSetAttribute(gain_gemm_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         PairCfg::SMEM);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2);
    cfg.blockDim = dim3(PairCfg::THREADS);
    cfg.dynamicSmemBytes = PairCfg::SMEM;
    return cudaOccupancyMaxActiveClusters(max_pairs, gain_gemm_pair_kernel, &cfg);
}

cudaError_t launch_gain_gemm_pair(const GemmArgs& a, cudaStream_t s) {
    const int grid = a.m_tiles * a.n_tiles * a.n_splits;  // m_tiles is even: grid pairs up
    return launch_pdl(gain_gemm_pair_kernel, dim3(grid), dim3(PairCfg::THREADS), (size_t)PairCfg::SMEM, s, a);
}

cudaError_t launch_gain_gemm(int bn, const GemmArgs& a, cudaStream_t s) {
    switch (bn) {
        case 64: return launch_gemm_bn<64>(a, s);
        case 128: return launch_gemm_bn<128>(a, s);
        case 256: return launch_gemm_bn<256>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

// ------------------------------------------------------------------ operand preparation
// One block per row: scale = 2^floor(log2(max |g|)) (1 for an all-zero row), then
// hi = bf16(g / scale), lo = bf16(g / scale - hi), written into the GEMM's tile-blocked layout:
// K tile t = cb * n1 + b holds G[r][b][64 cb .. 64 cb + 63] (zero past n2); tile (m, t) is
// 32 KB at ((m * T + t) * 2 + half) * 16 KB, row r % 128 at 128-byte pitch, and its 16-byte
// chunk q (elements 8q .. 8q + 7) stored at chunk q ^ (r % 8): the 128-byte swizzle that the
// UMMA descriptor expects of a 1024-byte aligned stage, so a flat bulk copy lands it ready.
__global__ void split_rows_kernel(const float* __restrict__ src, int row0, int n1, int n2, int n_cb,
                                  unsigned char* __restrict__ gt, float* row_scale) {
    __shared__ float s_max[256];
    const long long r = blockIdx.x;
    const float* g = src + (size_t)r * n1 * n2;
    float m = 0.f;
    for (long long k = threadIdx.x; k < (long long)n1 * n2; k += blockDim.x) m = fmaxf(m, fabsf(g[k]));
    s_max[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s_max[threadIdx.x] = fmaxf(s_max[threadIdx.x], s_max[threadIdx.x + o]);
        __syncthreads();
    }
    const float mx = s_max[0];
    int ex = 0;
    if (mx > 0.f && isfinite(mx)) frexpf(mx, &ex);  // mx = f * 2^ex, f in [0.5, 1)
    const float scale = ldexpf(1.f, ex - 1);         // mx / scale in [1, 2)
    const float inv = ldexpf(1.f, 1 - ex);
    if (threadIdx.x == 0) row_scale[r] = scale;
    const long long gr = row0 + r;  // stacked row of the group
    const long long T = (long long)n_cb * n1;
    const int rt = (int)(gr % kMmaM);
    unsigned char* rowbase = gt + (size_t)(gr / kMmaM) * T * kGTileBytes + (size_t)rt * 128;
    // one 16-byte chunk (8 elements) of hi and of lo per thread and iteration
    const long long chunks = (long long)n1 * n_cb * 8;
    for (long long q = threadIdx.x; q < chunks; q += blockDim.x) {
        const long long bt = q >> 3;           // (b, cb) pair
        const int cq = (int)(q & 7);           // chunk within the 64-wide block
        const long long b = bt / n_cb;
        const int cb = (int)(bt - b * n_cb);
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int c0 = cb * kMmaK + cq * 8 + 2 * e;
            const float v0 = c0 < n2 ? g[b * n2 + c0] * inv : 0.f;
            const float v1 = c0 + 1 < n2 ? g[b * n2 + c0 + 1] * inv : 0.f;
            const __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
            const __nv_bfloat162 hh = __halves2bfloat162(h0, h1);
            const __nv_bfloat162 ll = __halves2bfloat162(__float2bfloat16_rn(v0 - __bfloat162float(h0)),
                                                         __float2bfloat16_rn(v1 - __bfloat162float(h1)));
            h[e] = *reinterpret_cast<const uint32_t*>(&hh);
            l[e] = *reinterpret_cast<const uint32_t*>(&ll);
        }
        const long long t = (long long)cb * n1 + b;
        unsigned char* tile = rowbase + (size_t)t * kGTileBytes;
        const int phys = ((cq ^ (rt & 7)) << 4);
        *reinterpret_cast<uint4*>(tile + phys) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(tile + kGTileBytes / 2 + phys) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

cudaError_t launch_split_rows(const float* src, long long rows, int row0, int n1, int n2, int n_cb,
                              unsigned char* gt, float* row_scale, cudaStream_t s) {
    split_rows_kernel<<<(unsigned)rows, 256, 0, s>>>(src, row0, n1, n2, n_cb, gt, row_scale);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ batched Euler epilogue
namespace {


constexpr int kRT = 32;   // rows per tile
constexpr int kIT = 32;   // instances per tile
constexpr int kCK = kRowsChunk;  // K chunk of the loss / emission tile products
constexpr int kOP = kCK + 8;      // BF16 row pitch of a staged operand chunk (272 bytes: 16-byte
                                  // aligned rows whose 8-row ldmatrix phases hit 32 distinct banks)
constexpr int kFP = kIT + 4;      // FP32 row pitch of a staged state chunk (conflict-free B loads)
constexpr int kRowStages = 3;     // cp.async ring depth
constexpr int kOpBytes = kRT * kOP * 2;  // one half (hi or lo) of one operand chunk
constexpr int kStageBytes = 4 * kOpBytes + kCK * kFP * 4;  // loss hi, lo, emission hi, lo, state chunk
constexpr int kRowsSmem = kRowStages * kStageBytes;  // dynamic: the operand / state chunk ring


__device__ __forceinline__ int species_of_row(const MixedRowOps& ops, int a) {
    int s = 0;
    while (s + 1 < ops.n_species && a >= ops.sp_off[s + 1]) ++s;
    return s;
}

// Loss and emission of one (row, instance) pair with direct loads (tiles the fast path cannot take),
// from the same BF16 hi + lo operands as the tile products: each operand value hi + lo (exact in
// FP32) times the state in FP32, the row scale applied to the sum.
// a: state row (global), am: its momentum index within cell `cell`, s: its species.
__device__ void row_terms_direct(const MixedRowOps& ops, const float* __restrict__ F, int a, int am, int cell, int s,
                                 int i, float& loss, float& emi) {
    const int B = ops.Bcap;
    loss = 0.f;
    emi = 0.f;
    if (ops.has_bin) {
        const int la = am - ops.sp_off[s];
        for (int b = ops.loss_ptr[s]; b < ops.loss_ptr[s + 1]; ++b) {
            const __nv_bfloat16* row = ops.loss_data + ops.loss_data_off[b] + (size_t)la * ops.loss_ld[b];
            const int co = ops.loss_col_off[b] + cell * ops.n_mom, nc = ops.loss_ncols[b];
            for (int c = 0; c < nc; ++c)
                loss += (__bfloat162float(row[c]) + __bfloat162float(row[c + ops.loss_lo])) * F[(size_t)(co + c) * B + i];
        }
        loss *= ops.loss_rscale[am];
    }
    if (ops.has_emi) {
        for (int p = ops.emi_rptr[a]; p < ops.emi_rptr[a + 1]; ++p) {
            const int pc = ops.emi_piece[p];
            const __nv_bfloat16* row = ops.emi_data + ops.emi_data_off[pc] + (size_t)(a - ops.emi_row0[pc]) * ops.emi_ld[pc];
            const int col0 = ops.emi_col0[pc], nc = ops.emi_ncols[pc];
            for (int c = 0; c < nc; ++c)
                emi += (__bfloat162float(row[c]) + __bfloat162float(row[c + ops.emi_lo])) * F[(size_t)(col0 + c) * B + i];
        }
        emi *= ops.emi_rscale[a];
    }
}


// 16-byte asynchronous copy global -> shared; src_bytes 0 fills the destination with zeros.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// One 32-row x 32-instance tile per block, 512 threads. Loss and emission are tile products
// when the tile's rows belong to one species and every emission piece touching them covers
// them all (tile_fast): all their K chunks form one job list streamed through a 3-stage
// cp.async ring (operand chunk 32 x 128 as BF16 hi and lo halves, state chunk 128 x 32 FP32).
// The products run on the tensor cores as m16n8k16 BF16 MMAs with FP32 accumulation: each of
// the 16 warps owns a 16-row x 8-instance block over one half of every chunk's K range, splits
// the state into BF16 hi + lo as it builds its B fragments, and accumulates
// hi*hi + hi*lo + lo*hi (the scheme of the gain GEMM); the two K halves' sums are added in a
// fixed order and scaled back by the rows' power-of-two scales. The update then gives each
// thread one row and two instances, with every load it needs issued before the arithmetic
// (flux columns and values, state, vectors), so the latency of the L2 round trips overlaps.
constexpr int kRowsThreads = 512;
constexpr int kKHalves = 2;  // K halves of each product chunk (8 warps each)
static_assert(kRowsThreads / 32 == 2 * 4 * kKHalves, "16 warps: 2 row blocks x 4 instance blocks x 2 K halves");
static_assert((2 * kKHalves + 2) * kRT * (kIT + 1) * 4 <= kRowStages * kStageBytes,
              "the K halves' loss and emission tiles and the gather's half sums fit the ring");
constexpr int kEllFast = 8;  // ELL widths up to this take the hoisted-load flux path
constexpr int kGatherChunk = 18;  // split partials in flight per instance in the gain gather
constexpr int kGatherVec = 18;    // 16-byte split partials in flight per thread in the vector gather

__global__ void __launch_bounds__(kRowsThreads) mixed_rows_kernel(MixedRowOps ops, const float* __restrict__ F,
                                                                  const float* __restrict__ Cc,
                                                                  float* __restrict__ Fo, float* __restrict__ Co,
                                                                  const unsigned long long* gstep, int kpos) {
    __shared__ float s_gain[kRT][kIT + 1];
    __shared__ RowJob s_job[kRowsMaxJobs];
    __shared__ int s_njob;
    extern __shared__ __align__(16) float rows_dyn[];
    // after the products the same memory holds the two K halves' loss and emission tiles
    float(*s_pl)[kRT][kIT + 1] = reinterpret_cast<float(*)[kRT][kIT + 1]>(rows_dyn);
    float(*s_pe)[kRT][kIT + 1] = reinterpret_cast<float(*)[kRT][kIT + 1]>(rows_dyn + kKHalves * kRT * (kIT + 1));
    unsigned char* ring = reinterpret_cast<unsigned char*>(rows_dyn);
    __shared__ double s_min[kRT][kIT + 1];  // padded: the per-instance reduction reads down columns
    __shared__ int s_nonfin[kIT];
    const int tid = threadIdx.x;
    // products: warp w takes rows 16 (w & 1) .. + 15, instances 8 ((w >> 1) & 3) .. + 7 and the
    // K half w >> 3 of every chunk
    const int wp = tid >> 5, ln = tid & 31;
    const int mblk = wp & 1, nblk = (wp >> 1) & 3, khalf = wp >> 3;
    const int a0 = blockIdx.x * kRT, i0 = blockIdx.y * kIT;
    const int n = ops.n_state, B = ops.Bcap;
    // the device step counter advances once per launch sequence (advance_step); kpos is this
    // launch's place in the sequence
    const long long step = (long long)*reinterpret_cast<const volatile unsigned long long*>(gstep) + kpos;
    const bool fast = ops.tile_fast[blockIdx.x] != 0;

    if (fast) {  // the tile's product chunks (host-built job list)
        if (tid < kRowsMaxJobs) s_job[tid] = ops.jobs[(size_t)blockIdx.x * kRowsMaxJobs + tid];
        if (tid == 0) s_njob = ops.njobs[blockIdx.x];
    }
    // ---- update operands, loaded ahead of the products so their latency overlaps them
    const int r = tid >> 4;
    const int a = a0 + r;
    const int jb = (tid & 15) * 2;
    const int ib = i0 + jb;
    const bool mine = a < n && ib < B;
    const bool ell_fast = ops.ell_w <= kEllFast;
    float2 fa2 = make_float2(0.f, 0.f), ca2 = make_float2(0.f, 0.f);
    double inv_ap = 0.0, injv = 0.0;
    bool act[2] = {false, false};
    double dts[2] = {0.0, 0.0};
    int cols[kEllFast];
    float vals[kEllFast];
#pragma unroll
    for (int e = 0; e < kEllFast; ++e) {
        cols[e] = -1;
        vals[e] = 0.f;
    }
    float lsc = 1.f, esc = 1.f;
    if (mine) {
        inv_ap = (double)__ldg(ops.invAp + a);
        injv = (double)__ldg(ops.inj + a);
        if (ops.has_bin) lsc = __ldg(ops.loss_rscale + (a % ops.n_mom));
        if (ops.has_emi) esc = __ldg(ops.emi_rscale + a);
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int i = ib + j;
            act[j] = i < B && step < ops.stop_step[i];
            dts[j] = i < B ? ops.dt_scale[i] : 0.0;
        }
        if (ell_fast) {
            const int* crow = ops.ell_col + (size_t)a * ops.ell_w;
            const float* vrow = ops.ell_val + (size_t)a * ops.ell_w;
#pragma unroll
            for (int e = 0; e < kEllFast; ++e) {
                if (e < ops.ell_w) {
                    cols[e] = __ldg(crow + e);
                    vals[e] = __ldg(vrow + e);
                }
            }
        }
    }

    // Everything up to the gain gather reads only static operands and the state F, C of this
    // step, which the previous step's epilogue wrote before this step's GEMM passed its own wait
    // (and so before this grid could launch). The products and the update's loads therefore run
    // before this grid waits for the GEMM, on SMs as the GEMM's blocks leave them; only the
    // gather of the GEMM's split partials follows the wait.
    __syncthreads();  // the job table is visible
    // the next step's GEMM may launch now: it waits for this grid's completion before it reads
    // the new state, so only its set-up (barriers, tensor memory, its first G tile) overlaps
    if (tid == 0) pdl_trigger();
    // a chunk into ring stage st: 512 16-byte pieces of each operand half (32 rows x 128 BF16)
    // and 1024 of the state (128 rows x 32 FP32), 4 + 2 per thread
    auto issue = [&](int k, int st) {
        unsigned char* base = ring + (size_t)st * kStageBytes;
        const RowJob J = s_job[k];
        {
            const int rr = tid >> 4, c8 = (tid & 15) * 8;
            const bool ok = a0 + rr < n && J.c0 + c8 < J.nc;
            const size_t ol = (size_t)rr * kOP + c8;
            if (J.TL) {
                const __nv_bfloat16* src = J.TL + (size_t)rr * J.ldl + J.c0 + c8;
                cp_async16(base + 2 * ol, ok ? src : J.TL, ok ? 16 : 0);
                cp_async16(base + kOpBytes + 2 * ol, ok ? src + ops.loss_lo : J.TL, ok ? 16 : 0);
            }
            if (J.TE) {
                const __nv_bfloat16* src = J.TE + (size_t)rr * J.lde + J.c0 + c8;
                cp_async16(base + 2 * kOpBytes + 2 * ol, ok ? src : J.TE, ok ? 16 : 0);
                cp_async16(base + 3 * kOpBytes + 2 * ol, ok ? src + ops.emi_lo : J.TE, ok ? 16 : 0);
            }
        }
        float* sF = reinterpret_cast<float*>(base + 4 * kOpBytes);
#pragma unroll
        for (int q2 = 0; q2 < 2; ++q2) {
            const int q = tid + kRowsThreads * q2;
            const int cr = q >> 3, i4 = (q & 7) * 4;
            // state rows past the operand's columns are zero: the A operand there is zero too,
            // and zero times a stale value could be a NaN
            const bool okf = J.c0 + cr < J.nc && i0 + i4 < B;
            const float* srcf = okf ? F + (size_t)(J.col0 + J.c0 + cr) * B + i0 + i4 : F;
            cp_async16(sF + cr * kFP + i4, srcf, okf ? 16 : 0);
        }
    };
    // the first chunks are in flight while the update's operands are loaded below
    if (fast) {
#pragma unroll
        for (int k = 0; k < kRowStages - 1; ++k) {
            if (k < s_njob) issue(k, k);
            cp_async_commit();  // empty groups keep the group count uniform
        }
    }
    if (mine) {
        const size_t idx = (size_t)a * B + ib;  // B and ib are even
        fa2 = *reinterpret_cast<const float2*>(F + idx);
        ca2 = *reinterpret_cast<const float2*>(Cc + idx);
    }
    if (tid < kIT) s_nonfin[tid] = 0;
    __syncthreads();
    float2 fv[kEllFast];
#pragma unroll
    for (int e = 0; e < kEllFast; ++e)
        fv[e] = (mine && cols[e] >= 0) ? *reinterpret_cast<const float2*>(F + (size_t)cols[e] * B + ib)
                                       : make_float2(0.f, 0.f);

    // MMA accumulators of the warp's 16 x 8 block: rows g and g + 8, instances 2t and 2t + 1
    // (g = lane / 4, t = lane % 4)
    // (hi*hi and the hi*lo + lo*hi corrections in separate accumulators, as in the gain GEMM)
    float acc_l[4] = {0.f, 0.f, 0.f, 0.f}, acc_e[4] = {0.f, 0.f, 0.f, 0.f};
    float cor_l[4] = {0.f, 0.f, 0.f, 0.f}, cor_e[4] = {0.f, 0.f, 0.f, 0.f};
    if (fast) {
        const int nj = s_njob;
        const int g = ln >> 2, t = ln & 3;
        // ldmatrix row of this lane: matrices 0/1 take rows 0-7 / 8-15 at K 0-7, 2/3 at K 8-15
        const int lrow = 16 * mblk + (ln & 7) + ((ln >> 3) & 1) * 8, lcol = (ln >> 4) * 8;
        for (int k = 0; k < nj; ++k) {
            cp_async_wait<kRowStages - 2>();
            __syncthreads();  // chunk k landed for every thread; chunk k - 1's stage is free
            if (k + kRowStages - 1 < nj) issue(k + kRowStages - 1, (k + kRowStages - 1) % kRowStages);
            cp_async_commit();
            const unsigned char* base = ring + (size_t)(k % kRowStages) * kStageBytes;
            const uint32_t sa = smem_addr(base);
            const float* sF = reinterpret_cast<const float*>(base + 4 * kOpBytes);
            const bool hl = s_job[k].TL != nullptr, he = s_job[k].TE != nullptr;
#pragma unroll
            for (int kk = 0; kk < kCK / kKHalves / 16; ++kk) {
                const int kb = khalf * (kCK / kKHalves) + kk * 16;
                // B fragment: state rows kb + 2t, +1 and kb + 2t + 8, +9 of instance 8 nblk + g
                const float* fp = sF + (kb + 2 * t) * kFP + 8 * nblk + g;
                uint32_t bh0, bl0, bh1, bl1;
                split_pair(fp[0], fp[kFP], bh0, bl0);
                split_pair(fp[8 * kFP], fp[9 * kFP], bh1, bl1);
                const uint32_t ao = (uint32_t)(2 * (lrow * kOP + kb + lcol));
                if (hl) {
                    uint32_t ah[4], al[4];
                    ldsm_x4(sa + ao, ah);
                    ldsm_x4(sa + kOpBytes + ao, al);
                    mma_bf16_16816(acc_l, ah, bh0, bh1);
                    mma_bf16_16816(cor_l, ah, bl0, bl1);
                    mma_bf16_16816(cor_l, al, bh0, bh1);
                }
                if (he) {
                    uint32_t ah[4], al[4];
                    ldsm_x4(sa + 2 * kOpBytes + ao, ah);
                    ldsm_x4(sa + 3 * kOpBytes + ao, al);
                    mma_bf16_16816(acc_e, ah, bh0, bh1);
                    mma_bf16_16816(cor_e, ah, bl0, bl1);
                    mma_bf16_16816(cor_e, al, bh0, bh1);
                }
            }
        }
        cp_async_wait<0>();
        __syncthreads();  // the ring is free: park the K halves' sums
        const int r0 = 16 * mblk + g, c0 = 8 * nblk + 2 * t;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            acc_l[q] += cor_l[q];
            acc_e[q] += cor_e[q];
        }
        s_pl[khalf][r0][c0] = acc_l[0];
        s_pl[khalf][r0][c0 + 1] = acc_l[1];
        s_pl[khalf][r0 + 8][c0] = acc_l[2];
        s_pl[khalf][r0 + 8][c0 + 1] = acc_l[3];
        s_pe[khalf][r0][c0] = acc_e[0];
        s_pe[khalf][r0][c0 + 1] = acc_e[1];
        s_pe[khalf][r0 + 8][c0] = acc_e[2];
        s_pe[khalf][r0 + 8][c0 + 1] = acc_e[3];
    }
    pdl_wait();  // this step's gain GEMM has completed: its split partials are visible
    // ---- gain of the tile from the reduced group sums
    // Vector gather (tiles of one cell and species whose group rows start on a multiple of 4,
    // in groups of M a multiple of 4): the two halves of the block take the two halves of the
    // split range, each thread 4 consecutive rows of one instance with 16-byte loads, all of a
    // half's loads in flight at once (the scalar gather below needs two L2 round trips); each
    // half sums its splits in order, and the two half sums are added in a fixed order.
    bool vec_gain = false;
    if (ops.has_bin && fast) {
        const int cell = a0 / ops.n_mom, am0 = a0 - cell * ops.n_mom;
        const int s = species_of_row(ops, am0);
        vec_gain = a0 + kRT <= n;
        for (int e = ops.gain_ptr[s]; e < ops.gain_ptr[s + 1] && vec_gain; ++e) {
            const int gi = ops.gain_grp[e];
            vec_gain = ((ops.gain_roff[e] + am0 - ops.sp_off[s]) % 4 == 0) && (ops.grp_M[gi] % 4 == 0);
        }
    }
    if (vec_gain) {
        float(*s_half)[kRT][kIT + 1] =
            reinterpret_cast<float(*)[kRT][kIT + 1]>(rows_dyn + 2 * kKHalves * kRT * (kIT + 1));
        const int cell = a0 / ops.n_mom, am0 = a0 - cell * ops.n_mom;
        const int s = species_of_row(ops, am0);
        const bool on = ops.bin_on == nullptr || ops.bin_on[cell] != 0;
        const int h = tid >> 8, q = tid & 255, rg = q & 7, il = q >> 3;  // rows 4 rg .. + 3, instance il
        const bool okv = on && i0 + il < B;
        // the combine below: thread (row r, instances il0 and il0 + 16)
        const int r = tid & (kRT - 1), il0 = tid >> 5;
        float g0 = 0.f, g1 = 0.f;
        for (int e = ops.gain_ptr[s]; e < ops.gain_ptr[s + 1]; ++e) {
            const int gi = ops.gain_grp[e];
            const int row0 = ops.gain_roff[e] + (am0 - ops.sp_off[s]);
            const int Mg = ops.grp_M[gi];
            const int nsp = ops.grp_nsplit[gi];
            const int sp_lo = h == 0 ? 0 : (nsp + 1) / 2, sp_hi = h == 0 ? (nsp + 1) / 2 : nsp;
            const float* pp = ops.grp_partial[gi] + ((size_t)cell * B + i0 + il) * Mg + row0 + 4 * rg;
            const size_t st = (size_t)ops.grp_stride[gi];
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int c0 = sp_lo; c0 < sp_hi; c0 += kGatherVec) {
                float4 v[kGatherVec];
#pragma unroll
                for (int k = 0; k < kGatherVec; ++k)
                    v[k] = (okv && c0 + k < sp_hi) ? *reinterpret_cast<const float4*>(pp + (size_t)(c0 + k) * st)
                                                   : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int k = 0; k < kGatherVec; ++k) {
                    if (c0 + k < sp_hi) {
                        acc.x += v[k].x;
                        acc.y += v[k].y;
                        acc.z += v[k].z;
                        acc.w += v[k].w;
                    }
                }
            }
            s_half[h][4 * rg][il] = acc.x;
            s_half[h][4 * rg + 1][il] = acc.y;
            s_half[h][4 * rg + 2][il] = acc.z;
            s_half[h][4 * rg + 3][il] = acc.w;
            __syncthreads();
            const float rs = ops.grp_rscale[gi][row0 + r];
            if (on && i0 + il0 < B)
                g0 += (s_half[0][r][il0] + s_half[1][r][il0]) * rs * ops.grp_sig1[gi][i0 + il0] * ops.grp_sig2[gi][i0 + il0];
            if (on && i0 + il0 + 16 < B)
                g1 += (s_half[0][r][il0 + 16] + s_half[1][r][il0 + 16]) * rs * ops.grp_sig1[gi][i0 + il0 + 16] *
                      ops.grp_sig2[gi][i0 + il0 + 16];
            __syncthreads();  // s_half is reused by the next group
        }
        s_gain[r][il0] = g0;
        s_gain[r][il0 + 16] = g1;
    } else if (ops.has_bin) {
        const int r = tid & (kRT - 1);
        const int a = a0 + r;
        const int cell = a / ops.n_mom, am = a - cell * ops.n_mom;
        const int s = a < n ? species_of_row(ops, am) : 0;
        const bool on = a < n && (ops.bin_on == nullptr || ops.bin_on[cell] != 0);
        // the thread's two instances il0 and il0 + 16; their partials are loaded kGatherChunk
        // splits at a time for both instances at once (one L2 round trip per chunk), then summed
        // in split order
        const int il0 = tid >> 5;
        const bool ok0 = on && i0 + il0 < B, ok1 = on && i0 + il0 + 16 < B;
        float g0 = 0.f, g1 = 0.f;
        if (ok0 || ok1) {
            for (int e = ops.gain_ptr[s]; e < ops.gain_ptr[s + 1]; ++e) {
                const int gi = ops.gain_grp[e];
                const int row = ops.gain_roff[e] + (am - ops.sp_off[s]);
                const int Mg = ops.grp_M[gi];
                // column cell * Bcap + slot of the group's partials
                const float* pp0 = ops.grp_partial[gi] + ((size_t)cell * B + i0 + il0) * Mg + row;
                const float* pp1 = pp0 + (size_t)16 * Mg;
                const size_t st = (size_t)ops.grp_stride[gi];
                const int nsp = ops.grp_nsplit[gi];
                float acc0 = 0.f, acc1 = 0.f;
                for (int sp0 = 0; sp0 < nsp; sp0 += kGatherChunk) {
                    float v0[kGatherChunk], v1[kGatherChunk];
#pragma unroll
                    for (int k = 0; k < kGatherChunk; ++k) {
                        const bool in = sp0 + k < nsp;
                        v0[k] = (in && ok0) ? pp0[(size_t)(sp0 + k) * st] : 0.f;
                        v1[k] = (in && ok1) ? pp1[(size_t)(sp0 + k) * st] : 0.f;
                    }
#pragma unroll
                    for (int k = 0; k < kGatherChunk; ++k) {
                        if (sp0 + k < nsp) {
                            acc0 += v0[k];
                            acc1 += v1[k];
                        }
                    }
                }
                const float rs = ops.grp_rscale[gi][row];
                if (ok0) g0 += acc0 * rs * ops.grp_sig1[gi][i0 + il0] * ops.grp_sig2[gi][i0 + il0];
                if (ok1) g1 += acc1 * rs * ops.grp_sig1[gi][i0 + il0 + 16] * ops.grp_sig2[gi][i0 + il0 + 16];
            }
        }
        s_gain[r][il0] = g0;
        s_gain[r][il0 + 16] = g1;
    }
    __syncthreads();

    // ---- update: one row, two instances per thread
    double rmin[2] = {CUDART_INF, CUDART_INF};
    int nonfin[2] = {0, 0};
    if (mine) {
        const size_t idx = (size_t)a * B + ib;
        float flux[2] = {0.f, 0.f};
        if (ell_fast) {
#pragma unroll
            for (int e = 0; e < kEllFast; ++e) {
                if (cols[e] < 0) continue;  // padding: only stored entries take part
                flux[0] += vals[e] * fv[e].x;
                flux[1] += vals[e] * fv[e].y;
            }
        } else {
            const int* crow = ops.ell_col + (size_t)a * ops.ell_w;
            const float* vrow = ops.ell_val + (size_t)a * ops.ell_w;
            for (int e = 0; e < ops.ell_w; ++e) {
                const int col = __ldg(crow + e);
                if (col < 0) continue;
                const float v = __ldg(vrow + e);
                const float2 f2 = *reinterpret_cast<const float2*>(F + (size_t)col * B + ib);
                flux[0] += v * f2.x;
                flux[1] += v * f2.y;
            }
        }
        const int cell = a / ops.n_mom, am = a - cell * ops.n_mom;
        const int s = species_of_row(ops, am);
        // the binary term of this cell (SteppingMethods.jl:369-380): Vol of the cell, zero outside
        // BinM.Domain
        const bool bin_here = ops.has_bin && (ops.bin_on == nullptr || ops.bin_on[cell] != 0);
        const float vol = ops.vol_cell[cell];
        const float fa[2] = {fa2.x, fa2.y};
        const float ca[2] = {ca2.x, ca2.y};
        float fo[2], co[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if (!act[j]) {
                fo[j] = fa[j];
                co[j] = ca[j];
                continue;
            }
            float loss, emi;
            if (fast) {  // the K halves in a fixed order, then the rows' scales (powers of two)
                loss = (s_pl[0][r][jb + j] + s_pl[1][r][jb + j]) * lsc;
                emi = (s_pe[0][r][jb + j] + s_pe[1][r][jb + j]) * esc;
            } else {
                row_terms_direct(ops, F, a, am, cell, s, ib + j, loss, emi);
            }
            const float gain = ops.has_bin ? s_gain[r][jb + j] : 0.f;
            // SteppingMethods.jl:31-46 in FP32, the scaling in FP64
            float df = -flux[j];
            if (ops.has_emi) df += emi;
            if (ops.has_bin) df += bin_here ? vol * (gain - fa[j] * loss) : 0.f;
            const double dfs = (double)df * (inv_ap * dts[j]);
            // :97-101 with an FP64 compensated sum: the state is fa + ca
            double t = ((double)fa[j] + (double)ca[j]) + (dfs + injv * dts[j]);
            t = (t >= ops.thr) ? t : copysign(0.0, t);
            t = (t != CUDART_INF) ? t : copysign(0.0, t);
            fo[j] = (float)t;
            co[j] = (float)(t - (double)fo[j]);
            double ratio = dfs / (double)fa[j];
            if (isnan(ratio)) ratio = CUDART_INF;
            if (ratio < rmin[j] || (ratio == rmin[j] && signbit(ratio))) rmin[j] = ratio;
            if (!isfinite(dfs)) nonfin[j] = 1;
        }
        *reinterpret_cast<float2*>(Fo + idx) = make_float2(fo[0], fo[1]);
        *reinterpret_cast<float2*>(Co + idx) = make_float2(co[0], co[1]);
    }
    // ---- per-instance diagnostics over the tile's rows, then one atomic per instance
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        s_min[r][jb + j] = rmin[j];
        if (nonfin[j]) atomicOr(&s_nonfin[jb + j], 1);
    }
    __syncthreads();
    {
        // 16 lanes per instance, two rows each, then a shuffle tree (min with -0.0 below +0.0)
        const int il = tid >> 4, rg = tid & 15;
        double m = s_min[rg][il];
        const double v2 = s_min[rg + 16][il];
        if (v2 < m || (v2 == m && signbit(v2))) m = v2;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            const double v = __shfl_xor_sync(0xffffffffu, m, o);
            if (v < m || (v == m && signbit(v))) m = v;
        }
        const int i = i0 + il;
        if (rg == 0 && i < B && step < ops.stop_step[i]) {
            atomicMin(&ops.min_ratio[i], ord_enc(m));
            if (s_nonfin[il]) atomicOr(&ops.nonfinite[i], 1);
        }
    }
}

}  // namespace

// Per (slot, species) FP64 number sum(f) and energy sum(f * w) of the compensated state F + C
// (DistributionMoments.jl:33,145,162); out[(slot * n_species + s) * 2 + {0, 1}].
__global__ void batch_moments_kernel(const float* __restrict__ F, const float* __restrict__ C, int Bcap,
                                     const int* __restrict__ sp_off, int n_species, int n_mom,
                                     const double* __restrict__ w, double* __restrict__ out) {
    __shared__ double s_n[128], s_e[128];
    const int sp = blockIdx.x, slot = blockIdx.y, cell = blockIdx.z;
    double a = 0.0, e = 0.0;
    const size_t row0 = (size_t)cell * n_mom;
    for (int k = sp_off[sp] + threadIdx.x; k < sp_off[sp + 1]; k += blockDim.x) {
        const double v = (double)F[(row0 + k) * Bcap + slot] + (double)C[(row0 + k) * Bcap + slot];
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
    if (threadIdx.x == 0) {  // out[slot][cell][species][number, energy]
        const size_t o = (((size_t)slot * gridDim.z + cell) * n_species + sp) * 2;
        out[o + 0] = s_n[0];
        out[o + 1] = s_e[0];
    }
}

// Whole-batch state I/O: the user's slot-major f64 [Buser][n] <-> the slot-minor FP32 pair
// (F, C) [n][Bcap], F = fl32(v), C = fl32(v - F), through 32 x 32 shared-memory transposes so
// both sides are coalesced. Padding slots [Buser, Bcap) are written as zeros.
__global__ void __launch_bounds__(256) pack_f_kernel(const double* __restrict__ io, int Buser, int n, int Bcap,
                                                     float* __restrict__ F, float* __restrict__ C) {
    __shared__ double t[32][33];
    const int a0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = ty; k < 32; k += 8) {
        const int i = i0 + k, a = a0 + tx;
        t[k][tx] = (i < Buser && a < n) ? io[(size_t)i * n + a] : 0.0;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int a = a0 + k, i = i0 + tx;
        if (a < n && i < Bcap) {
            const double v = t[tx][k];
            const float fv = __double2float_rn(v);
            F[(size_t)a * Bcap + i] = fv;
            C[(size_t)a * Bcap + i] = __double2float_rn(__dsub_rn(v, (double)fv));
        }
    }
}

__global__ void __launch_bounds__(256) unpack_f_kernel(const float* __restrict__ F, const float* __restrict__ C,
                                                       int Buser, int n, int Bcap, double* __restrict__ io) {
    __shared__ double t[32][33];
    const int a0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = ty; k < 32; k += 8) {
        const int a = a0 + k, i = i0 + tx;
        t[k][tx] = (a < n && i < Buser) ? __dadd_rn((double)F[(size_t)a * Bcap + i], (double)C[(size_t)a * Bcap + i])
                                        : 0.0;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int i = i0 + k, a = a0 + tx;
        if (i < Buser && a < n) io[(size_t)i * n + a] = t[tx][k];
    }
}

cudaError_t launch_pack_f(const double* io, int Buser, int n, int Bcap, float* F, float* C, cudaStream_t s) {
    pack_f_kernel<<<dim3((n + 31) / 32, (Bcap + 31) / 32), 256, 0, s>>>(io, Buser, n, Bcap, F, C);
    return cudaGetLastError();
}

cudaError_t launch_unpack_f(const float* F, const float* C, int Buser, int n, int Bcap, double* io, cudaStream_t s) {
    unpack_f_kernel<<<dim3((n + 31) / 32, (Buser + 31) / 32), 256, 0, s>>>(F, C, Buser, n, Bcap, io);
    return cudaGetLastError();
}

cudaError_t launch_batch_moments(const float* F, const float* C, int Bcap, const int* sp_off, int n_species,
                                 int n_mom, int n_space, const double* w, double* out, cudaStream_t s) {
    batch_moments_kernel<<<dim3(n_species, Bcap, n_space), 128, 0, s>>>(F, C, Bcap, sp_off, n_species, n_mom, w, out);
    return cudaGetLastError();
}

__global__ void advance_step_kernel(unsigned long long* gstep, int n) { *gstep += (unsigned long long)n; }

// Admission of one slot from a staged record (f column, compensation column, the species
// scales and their reciprocals, dt / dt0, stop step): one launch instead of a copy per field.
__global__ void __launch_bounds__(256) admit_slot_kernel(const unsigned char* __restrict__ rec, int n, int ns, int slot,
                                                         int Bst, float* __restrict__ F, float* __restrict__ C,
                                                         float* __restrict__ sig, float* __restrict__ isig,
                                                         double* __restrict__ dt_scale, long long* __restrict__ stop,
                                                         unsigned long long* __restrict__ min_ratio,
                                                         int* __restrict__ nonfinite, unsigned long long inf_enc) {
    const AdmitRecord R = admit_record(n, ns);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        F[(size_t)i * Bst + slot] = reinterpret_cast<const float*>(rec + R.f)[i];
        C[(size_t)i * Bst + slot] = reinterpret_cast<const float*>(rec + R.c)[i];
    }
    if (i < ns) {
        sig[(size_t)i * Bst + slot] = reinterpret_cast<const float*>(rec + R.sig)[i];
        isig[(size_t)i * Bst + slot] = reinterpret_cast<const float*>(rec + R.isig)[i];
    }
    if (i == 0) {
        dt_scale[slot] = *reinterpret_cast<const double*>(rec + R.dt);
        stop[slot] = *reinterpret_cast<const long long*>(rec + R.stop);
        min_ratio[slot] = inf_enc;
        nonfinite[slot] = 0;
    }
}

cudaError_t launch_admit_slot(const unsigned char* rec, int n, int ns, int slot, int Bst, float* F, float* C, float* sig,
                              float* isig, double* dt_scale, long long* stop, unsigned long long* min_ratio,
                              int* nonfinite, unsigned long long inf_enc, cudaStream_t s) {
    const int th = std::max(n, ns);
    admit_slot_kernel<<<(th + 255) / 256, 256, 0, s>>>(rec, n, ns, slot, Bst, F, C, sig, isig, dt_scale, stop,
                                                       min_ratio, nonfinite, inf_enc);
    return cudaGetLastError();
}

cudaError_t launch_advance_step(unsigned long long* gstep, int n, cudaStream_t s) {
    advance_step_kernel<<<1, 1, 0, s>>>(gstep, n);
    return cudaGetLastError();
}

cudaError_t launch_mixed_rows(const MixedRowOps& ops, const float* F_in, const float* C_in, float* F_out, float* C_out,
                              const unsigned long long* gstep, int kpos, cudaStream_t s) {
    dim3 grid((ops.n_state + kRT - 1) / kRT, (ops.Bcap + kIT - 1) / kIT);
    return launch_pdl(mixed_rows_kernel, grid, dim3(kRowsThreads), (size_t)kRowsSmem, s, ops, F_in, C_in, F_out, C_out,
                      gstep, kpos);
}


int mixed_rows_tile_rows() { return kRT; }

cudaError_t prepare_mixed_rows() {
    return cudaFuncSetAttribute(mixed_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowsSmem);
}

}  // namespace dtb
