// Mixed-precision Schur update on the 5th-generation tensor cores (sm_100a).
//
//     C(rows, cols) -= (L D)(rows, K) * L(cols, K)'        (LMMY18, lmmy18.f:5-192)
//
// as 3xTF32 split products: x = hi + lo with hi = tf32(x), lo = tf32(x - hi),
// and A*B ~ A_lo*B_hi + A_hi*B_lo + A_hi*B_hi accumulated in FP32 in tensor
// memory over 256-column chunks, FP64 across chunks.  The mixed mode runs the
// K = S updates and the trailing-update columns beyond the next super-panel
// here; the updates inside the panel chain stay on the FP64 kernel.
//
// Two kernels per Schur-update launch:
//   k_split_tc  reads the FP64 panel columns [k_lo, k_hi) of rows [c0, r_end)
//               of each front and writes four K-major FP32 slabs (W_hi, W_lo,
//               L_hi, L_lo; W = L D) of 32-column blocks, [row][32] floats, rows
//               padded to a multiple of 128 and K to a multiple of 32 with
//               zeros, into the slab arena (one 128-byte row per slab row);
//   k_gemm_tc   persistent CTAs over the lower 128x128 tiles of the update
//               block: a TMA producer warp streams the four 128x32 operand
//               tiles of each K block into a 3-stage shared-memory ring
//               (128-byte swizzle), one thread issues tcgen05.mma kind::tf32
//               (M=N=128, K=8) into two alternating 128-column TMEM
//               accumulators and releases stages with tcgen05.commit, and four
//               epilogue warps add each chunk into FP64 sums kept in TMEM and
//               subtract the last one from the FP64 front (lower triangle only:
//               the upper triangle of diagonal blocks holds L11^-1 of later panels).
// Every mbarrier wait is bounded by a time limit; a wait that gives up sets
// Stats::tc_timeout, the CTA skips its remaining work, frees its TMEM and
// returns (the host turns the flag into an error).
#pragma once
#include <cuda.h>

namespace tc {

constexpr int kTM = 128;                  // M = N of the tile and of the MMA
constexpr int kBK = 32;                     // K block: 32 fp32 = one 128-byte swizzle row
constexpr int kStages = 3;
constexpr int kOperandBytes = kTM * kBK * 4;          // 16 KB: one 128x32 fp32 tile
constexpr int kStageBytes = 4 * kOperandBytes;           // A_hi, A_lo, B_hi, B_lo
constexpr size_t kSmem = (size_t)kStages * kStageBytes + 1024 + 256;
constexpr int kThreads = 192;               // warp 0 TMA, warp 1 MMA + TMEM owner, warps 2-5 epilogue
constexpr uint32_t kTmemCols = 512;       // FP32 accumulator pair [0,256) + FP64 sums [256,512)
constexpr int kChunk = 8;                   // K blocks (256 columns) per FP32 accumulation

// instruction descriptor: D f32, A/B tf32, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTM >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
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

// Bounded wait for the phase of the given parity; false when it gave up
// after limit_ns (PV::wait_ns, 2 s by default).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    for (;;) {
        for (int i = 0; i < 64; ++i)
            if (mbar_try(bar, parity)) return true;
        if (now_ns() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(dst),
        "l"(map), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

// K-major operand tile, 128-byte swizzle: 8-row groups 1024 B apart (SBO),
// descriptor version 1 (sm_100), layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 lanes x 32 consecutive 32-bit columns: thread t receives lane t's columns.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]),
        "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
        "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ int64_t padded_rows(const Job& jb) {
    return ((int64_t)(jb.r_end - jb.c0) + kTM - 1) / kTM * kTM;
}
__device__ __forceinline__ int k_blocks(const Job& jb) { return (jb.k_hi - jb.k_lo + kBK - 1) / kBK; }

// Lower tiles (it >= jt) of an nr x nct tile grid in groups of kGroup
// column tiles: inside a group the order is row by row, so the CTAs that run
// together share a few row panels (A) and a few column panels (B) and the
// operand slabs are served from L2 instead of HBM.
#ifndef SPR_TC_GROUP
#define SPR_TC_GROUP 8
#endif
constexpr int kGroup = SPR_TC_GROUP;
__device__ __forceinline__ void tile_of(int64_t u, int nct, int nr, int& it, int& jt) {
    int g0 = 0;
    for (;;) {
        const int w = min(kGroup, nct - g0);
        const int64_t tri = (int64_t)w * (w - 1) / 2;
        const int64_t cnt = tri + (int64_t)(nr - g0 - (w - 1)) * w;
        if (u < cnt || g0 + w >= nct) {
            if (u < tri) {
                int a = (int)((sqrt(8.0 * (double)u + 1.0) - 1.0) * 0.5);
                while ((int64_t)(a + 1) * (a + 2) / 2 <= u) ++a;
                while ((int64_t)a * (a + 1) / 2 > u) --a;
                it = g0 + a;
                jt = g0 + (int)(u - (int64_t)a * (a + 1) / 2);
            } else {
                const int64_t v = u - tri;
                it = g0 + (w - 1) + (int)(v / w);
                jt = g0 + (int)(v % w);
            }
            return;
        }
        u -= cnt;
        g0 += w;
    }
}

}  // namespace tc

// Split kernel: one CTA (256 threads) per 32-row x 32-column block of a job's
// panel; the transpose goes through shared memory so that both the FP64
// reads (column-major front) and the FP32 slab writes (row-major) coalesce.
__global__ void __launch_bounds__(256) k_split_tc(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P,
                                                   float* slab) {
    __shared__ float sw[2][32][33];
    __shared__ float sl[2][32][33];
    if (P.st->any_fail) return;
    const int64_t task = blockIdx.x;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (P.sn_bad[js] || node_off(P, js)) return;
    const int64_t np = tc::padded_rows(jb);
    const int nkb = tc::k_blocks(jb);
    const int64_t u = task - jb.task0;
    const int kb = (int)(u % nkb);
    const int rb = (int)(u / nkb);
    const int ld = P.buf_ld[js];
    const double* front = P.arena + P.buf_off[js];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    // read: thread (tx = row, ty + 8 q = column)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int kc = ty + 8 * q;
        const int k = jb.k_lo + kb * tc::kBK + kc;
        const int r = jb.c0 + rb * 32 + tx;
        double l = 0.0, d = 0.0;
        if (k < jb.k_hi && r < jb.r_end) {
            l = front[(int64_t)k * ld + r];
            d = front[(int64_t)k * (ld + 1)];
        }
        const double w = l * d;
        const float wh = tc::to_tf32((float)w), lh = tc::to_tf32((float)l);
        sw[0][kc][tx] = wh;
        sw[1][kc][tx] = tc::to_tf32((float)(w - (double)wh));
        sl[0][kc][tx] = lh;
        sl[1][kc][tx] = tc::to_tf32((float)(l - (double)lh));
    }
    __syncthreads();
    // write: thread (tx = column, ty + 8 q = row); slab a at row base
    // jb.slab + (a * nkb + kb) * np
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int rr = ty + 8 * q;
        const int64_t row = (int64_t)rb * 32 + rr;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const float v = a < 2 ? sw[a][tx][rr] : sl[a - 2][tx][rr];
            slab[(jb.slab + ((int64_t)a * nkb + kb) * np + row) * tc::kBK + tx] = v;
        }
    }
}

// Persistent: CTA b takes the tasks b, b + gridDim.x, ...; the stage ring and
// the accumulator pair run on across tiles, so the epilogue of one tile
// overlaps the MMAs of the next.  The FP32 accumulation runs over chunks of
// kChunk K blocks; between chunks the epilogue warps add the chunk into FP64
// partial sums kept in tensor memory, and the last chunk goes to the front.
__global__ void __launch_bounds__(tc::kThreads, 1)
    k_gemm_tc(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks, PV P,
              const __grid_constant__ CUtensorMap tm) {
    using namespace tc;
    extern __shared__ uint8_t tc_raw[];
    __shared__ uint64_t bars[2 * kStages + 5];
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    if (P.st->any_fail) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = (smem_u32(tc_raw) + 1023u) & ~1023u;
    const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[kStages]);
    const uint32_t accf0 = smem_u32(&bars[2 * kStages]), acce0 = smem_u32(&bars[2 * kStages + 2]);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(accf0 + 8 * b, 1);
            mbar_init(acce0 + 8 * b, 4);                  // one arrival per epilogue warp
        }
        mbar_init(smem_u32(&bars[2 * kStages + 4]), 1);   // MMA drain before the TMEM is freed
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---- TMA producer: K blocks of every tile, continuing ring position
        int64_t g = 0;
        for (int64_t task = blockIdx.x; task < ntasks && !*(volatile int*)&failed; task += gridDim.x) {
            const Job& jb = job_of(jobs, njobs, tmap, task);
            if (P.sn_bad[jb.node] || node_off(P, jb.node)) continue;
            int it, jt;
            tile_of(task - jb.task0, (jb.c_end - jb.c0 + kTM - 1) / kTM, (jb.r_end - jb.c0 + kTM - 1) / kTM, it, jt);
            const int64_t np = padded_rows(jb);
            const int nkb = k_blocks(jb);
            const int64_t ya = jb.slab + (int64_t)it * kTM, yb = jb.slab + (int64_t)jt * kTM;
            for (int kb = 0; kb < nkb; ++kb, ++g) {
                const int s = (int)(g % kStages);
                const uint32_t ph = (uint32_t)(g / kStages) & 1u;
                if (g >= kStages && !mbar_wait(empty0 + 8 * s, ph ^ 1u, P.wait_ns)) {
                    failed = 1;
                    break;
                }
                const uint32_t st = base + (uint32_t)s * kStageBytes;
                const uint32_t fb = full0 + 8 * s;
                if (P.tc_drop && blockIdx.x == 0 && g == 0) continue;     // watchdog test: never loaded
                mbar_expect_tx(fb, kStageBytes);
                const int64_t off = (int64_t)kb * np, arr = (int64_t)nkb * np;
                tma_load_2d(st, &tm, fb, 0, (int)(ya + off));                                  // W_hi
                tma_load_2d(st + kOperandBytes, &tm, fb, 0, (int)(ya + off + arr));               // W_lo
                tma_load_2d(st + 2 * kOperandBytes, &tm, fb, 0, (int)(yb + off + 2 * arr));       // L_hi
                tma_load_2d(st + 3 * kOperandBytes, &tm, fb, 0, (int)(yb + off + 3 * arr));       // L_lo
            }
        }
        // drain: the last kStages issued stages must have landed before exit
        for (int64_t q = (g > kStages ? g - kStages : 0); q < g; ++q)
            mbar_wait(full0 + 8 * (int)(q % kStages), (uint32_t)(q / kStages) & 1u, P.wait_ns);
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer: chunks of kChunk K blocks into alternating accumulators
        int64_t g = 0, h = 0;
        for (int64_t task = blockIdx.x; task < ntasks; task += gridDim.x) {
            const Job& jb = job_of(jobs, njobs, tmap, task);
            if (P.sn_bad[jb.node] || node_off(P, jb.node)) continue;
            const int nkb = k_blocks(jb);
            bool stop = false;
            for (int c0 = 0; c0 < nkb && !stop; c0 += kChunk, ++h) {
                const int b = (int)(h & 1);
                const int64_t use = h >> 1;
                if (use >= 1 && !mbar_wait(acce0 + 8 * b, (uint32_t)((use - 1) & 1), P.wait_ns)) {
                    failed = 1;
                    stop = true;
                    break;
                }
                fence_after_sync();
                const uint32_t acc = tmem + (uint32_t)(b * kTM);
                const int c1 = min(nkb, c0 + kChunk);
                for (int kb = c0; kb < c1; ++kb, ++g) {
                    const int s = (int)(g % kStages);
                    if (!mbar_wait(full0 + 8 * s, (uint32_t)(g / kStages) & 1u, P.wait_ns) ||
                        *(volatile int*)&failed) {
                        failed = 1;
                        stop = true;
                        break;
                    }
                    fence_after_sync();
                    const uint32_t st = base + (uint32_t)s * kStageBytes;
                    const uint64_t ah = sw128_desc(st), al = sw128_desc(st + kOperandBytes);
                    const uint64_t bh = sw128_desc(st + 2 * kOperandBytes), bl = sw128_desc(st + 3 * kOperandBytes);
#pragma unroll
                    for (int kk = 0; kk < kBK / 8; ++kk) {
                        const uint64_t adv = (uint64_t)(kk * 32) >> 4;     // 8 tf32 = 32 bytes along K
                        mma_tf32(acc, al + adv, bh + adv, (kb != c0 || kk != 0) ? 1u : 0u);
                        mma_tf32(acc, ah + adv, bl + adv, 1u);
                        mma_tf32(acc, ah + adv, bh + adv, 1u);
                    }
                    mma_commit(empty0 + 8 * s);
                }
                mma_commit(accf0 + 8 * b);      // arrives when this chunk's MMAs are done
            }
            if (stop) break;
        }
        // every MMA this thread issued has completed before the TMEM is freed
        // (after a timeout some may still be in flight without a commit)
        mma_commit(smem_u32(&bars[2 * kStages + 4]));
        if (!mbar_wait(smem_u32(&bars[2 * kStages + 4]), 0u, P.wait_ns)) failed = 1;
    } else if (warp >= 2) {
        // ---- epilogue: warp w owns TMEM lanes 32 (w % 4) .. + 31 (tile rows)
        const int q = warp & 3;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * q) << 16);
        int64_t h = 0;
        for (int64_t task = blockIdx.x; task < ntasks; task += gridDim.x) {
            const Job& jb = job_of(jobs, njobs, tmap, task);
            const int js = jb.node;
            if (P.sn_bad[js] || node_off(P, js)) continue;
            int it, jt;
            tile_of(task - jb.task0, (jb.c_end - jb.c0 + kTM - 1) / kTM, (jb.r_end - jb.c0 + kTM - 1) / kTM, it, jt);
            const int i0 = jb.c0 + it * kTM, j0 = jb.c0 + jt * kTM;
            const int nkb = k_blocks(jb);
            const int nch = (nkb + kChunk - 1) / kChunk;
            const int r = i0 + 32 * q + lane;
            const int ld = P.buf_ld[js];
            double* front = P.arena + P.buf_off[js];
            bool stop = false;
            for (int c = 0; c < nch; ++c, ++h) {
                const int b = (int)(h & 1);
                if (!mbar_wait(accf0 + 8 * b, (uint32_t)((h >> 1) & 1), P.wait_ns) || *(volatile int*)&failed) {
                    failed = 1;
                    stop = true;
                    break;
                }
                fence_after_sync();
                const uint32_t acc = lane_base + (uint32_t)(b * kTM);
                const uint32_t acc64 = lane_base + (uint32_t)(2 * kTM);
                for (int cc = 0; cc < kTM / 32; ++cc) {
                    uint32_t v[32];
                    tmem_ld32(acc + (uint32_t)(32 * cc), v);
                    double sum[32];
                    if (c == 0) {
#pragma unroll
                        for (int t = 0; t < 32; ++t) sum[t] = (double)__uint_as_float(v[t]);
                    } else {
                        uint32_t w0[32], w1[32];
                        tmem_ld32(acc64 + (uint32_t)(64 * cc), w0);
                        tmem_ld32(acc64 + (uint32_t)(64 * cc + 32), w1);
#pragma unroll
                        for (int t = 0; t < 16; ++t) {
                            sum[t] = __hiloint2double((int)w0[2 * t + 1], (int)w0[2 * t]) +
                                     (double)__uint_as_float(v[t]);
                            sum[16 + t] = __hiloint2double((int)w1[2 * t + 1], (int)w1[2 * t]) +
                                          (double)__uint_as_float(v[16 + t]);
                        }
                    }
                    if (c + 1 < nch) {
                        // keep the FP64 partial sums in TMEM (two 32-bit columns each)
                        uint32_t w0[32], w1[32];
#pragma unroll
                        for (int t = 0; t < 16; ++t) {
                            w0[2 * t] = (uint32_t)__double2loint(sum[t]);
                            w0[2 * t + 1] = (uint32_t)__double2hiint(sum[t]);
                            w1[2 * t] = (uint32_t)__double2loint(sum[16 + t]);
                            w1[2 * t + 1] = (uint32_t)__double2hiint(sum[16 + t]);
                        }
                        tmem_st32(acc64 + (uint32_t)(64 * cc), w0);
                        tmem_st32(acc64 + (uint32_t)(64 * cc + 32), w1);
                    } else if (r < jb.r_end) {
                        // all loads of the chunk first (independent), then the stores
                        double cv[32];
                        const double* src = front + (int64_t)r + (int64_t)(j0 + 32 * cc) * ld;
#pragma unroll
                        for (int t = 0; t < 32; ++t) {
                            const int col = j0 + 32 * cc + t;
                            cv[t] = (col < jb.c_end && r >= col) ? __ldcg(src + (int64_t)t * ld) : 0.0;
                        }
#pragma unroll
                        for (int t = 0; t < 32; ++t) {
                            const int col = j0 + 32 * cc + t;
                            if (col < jb.c_end && r >= col) front[(int64_t)r + (int64_t)col * ld] = cv[t] - sum[t];
                        }
                    }
                }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                fence_before_sync();
                __syncwarp();
                if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acce0 + 8 * b) : "memory");
            }
            if (stop) break;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && failed) atomicExch(&P.st->tc_timeout, 1);
    if (warp == 1) {
        fence_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}
