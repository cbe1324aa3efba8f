// Ozaki-scheme DGEMM on INT8 tensor cores, and SGEMM as a 3xBF16 split product.
//
// DGEMM by error-free splitting (Ozaki, Ogita, Oishi, Rump 2012; integer
// variant Ootomo, Ozaki, Yokota 2024), restated from the mathematics:
//
//   op(A)[i,p] = 2^{e_i} * (sum_{t=1..s} 2^{-7t} A_t[i,p] + r_ip),  |r_ip| < 2^{-7s}
//   op(B)[p,j] = 2^{f_j} * (sum_{u=1..s} 2^{-7u} B_u[p,j] + r'_pj)
//
// with e_i / f_j the binary exponents of the row / column maxima (so the
// scaled values lie in (-1, 1)) and A_t, B_u int8 digits in [-127, 127]
// produced by exact FP64 steps y <- 128 y, d = trunc(y), y <- y - d.  Then
//
//   C ~= sum_{g=2..s+1} 2^{e_i + f_j - 7g} * D_g,   D_g = sum_{t+u=g} A_t B_u
//
// Every D_g is an exact INT32 tensor-core product (|D_g| <= s k 127^2 is kept
// below 2^31 by splitting K into segments).  FP64 is used only for the
// exponent scan, the digit extraction and the recombination of the D_g.
//
// Kernels:
//   ozaki_absmax     row / column max |x| (bit patterns, atomicMax)       HBM-bound
//   ozaki_split      exponents + s int8 digit planes, K-major, padded    HBM-bound
//   umma_slice_gemm  persistent tcgen05 GEMM: TMA -> smem ring -> UMMA
//                    (kind::i8, INT32 accumulators in TMEM, two 256-column
//                    buffers) -> epilogue warps scale D_g to FP64 and
//                    accumulate into C (alpha, beta, ldc)                 tensor-bound
//
// 3xBF16 SGEMM: x = hi + lo (hi = bf16(x), lo = bf16(x - hi)) and
// C ~= hi_A hi_B + hi_A lo_B + lo_A hi_B, one FP32 TMEM accumulator
// (kind::f16 with BF16 inputs), same GEMM kernel with a FP32 epilogue.
//
// Replaces, for the GPU, the reference's dense real GEMM body
// (kernels/shared/matrix_matrix/packed_simd.zig:306) when the Ozaki method is
// selected; argument semantics are those of gemm.zig:1392.
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "bounded_wait.cuh"
#include "common.cuh"
#include "kernels.h"
#include "ozaki.h"

namespace zb {
namespace {

// ------------------------------------------------------------ geometry
constexpr int kUM = 128;          // C rows per tile (TMEM lanes)
constexpr int kUN = 256;          // C columns per tile (TMEM columns per accumulator)
constexpr int kChunkBytes = 128;  // K bytes per operand chunk (one 128-byte swizzle row)
constexpr int kASlots = 4;        // ring of A digit chunks (128 x 128 B each)
constexpr int kBSlots = 4;        // ring of B digit chunks (256 x 128 B each)
constexpr int kAChunk = kUM * kChunkBytes;  // 16 KB
constexpr int kBChunk = kUN * kChunkBytes;  // 32 KB
constexpr int kThreads = 192;               // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int kMaxSteps = 96;
constexpr int kMaxJobs = 16;
constexpr size_t kSmemBytes = 1024 /*align slack*/ + kASlots * kAChunk + kBSlots * kBChunk + 256 + kUN * 8 + 3 * kMaxSteps;

enum Kind : int { KIND_I8 = 0, KIND_BF16 = 1 };
enum Epi : int { EPI_OZAKI_F64 = 0, EPI_F32 = 1, EPI_RESIDUE = 2 };

// Work of one C tile is a list of "group jobs".  A job owns one or two
// accumulators (TMEM columns [0,256) and [256,512)); it sweeps K chunk by
// chunk and, for every chunk, walks its steps (digit pairs).  Consecutive
// steps are ordered so that they share the A or the B digit chunk, which is
// then loaded once and used twice.
struct UmmaParams {
    int m, n;            // C extent
    int m_pad, n_pad;    // rows per plane of the A / B digit tensors
    int k_chunks;        // total K chunks
    int kseg_chunks;     // K chunks per accumulation segment (INT32 overflow bound)
    int num_kseg;
    int tiles_m, tiles_n, num_tiles;
    int num_jobs;
    int job_first_step[kMaxJobs];
    int job_num_steps[kMaxJobs];
    int job_groups[kMaxJobs];     // 1 or 2 accumulators
    int job_shift[kMaxJobs][2];   // 7 g of the group held by accumulator 0 / 1 (EPI_RESIDUE: modulus index)
    int job_buf[kMaxJobs];        // EPI_RESIDUE: TMEM accumulator (0 / 1) of the job
    int step_a[kMaxSteps];        // digit plane of A
    int step_b[kMaxSteps];        // digit plane of B
    int step_acc[kMaxSteps];      // accumulator 0 / 1
    double alpha, beta;
    float alpha_f, beta_f;
    void* c;
    long ldc;
    const int* row_exp;
    const int* col_exp;
    int* status;
    int8_t* residues;  // EPI_RESIDUE: residue planes [modulus][m_pad][n_pad] (row-major)
    long res_plane;
    int band_rows;     // EPI_RESIDUE on the CTA pair: tile-rows per raster band
    int tri;           // EPI_RESIDUE on the CTA pair: 1 / 2 = only the tiles meeting the upper / lower
                       // triangle (num_tiles of them, tiles_m == tiles_n), enumerated by crt_job_tile
    int* report;       // per-device report word of bounded waits that ran out
    unsigned long long wait_ns;  // time limit of every mbarrier wait
    int hold;          // test-only: the MMA issuer first waits on a barrier nothing arrives on
};

ZB_DEVICE void tile_coords(int tile, int tiles_m, int tiles_n, int& tm, int& tn, int G = 8) {
    // Bands of G tile-rows sweep the tile-columns, so CTAs running together
    // share A row blocks and B column blocks in L2.
    int band = tile / (G * tiles_n);
    int rows_in_band = min(G, tiles_m - band * G);
    int r = tile - band * G * tiles_n;
    tm = band * G + r % rows_in_band;
    tn = r / rows_in_band;
}

// Tile of CRT job index `tile`: the raster bands of tile_coords, or in triangle
// mode the T (T + 1) / 2 tiles meeting the stored triangle (rows <= columns for
// tri = 1, >= for tri = 2), row after row of the triangle: index t lies in
// triangle row r = floor((sqrt(8 t + 1) - 1) / 2) at position t - r (r + 1) / 2.
ZB_DEVICE void crt_job_tile(int tri, int tile, int tiles_m, int tiles_n, int band_rows, int& tm, int& tn) {
    if (!tri) {
        tile_coords(tile, tiles_m, tiles_n, tm, tn, band_rows);
        return;
    }
    int r = (int)((sqrt(8.0 * tile + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= tile) ++r;  // exact integer fix-up of the FP64 estimate
    while (r * (r + 1) / 2 > tile) --r;
    const int pos = tile - r * (r + 1) / 2;
    if (tri == 2) {  // lower: row r of tiles, columns 0 .. r
        tm = r;
        tn = pos;
    } else {  // upper: column r of tiles, rows 0 .. r
        tn = r;
        tm = pos;
    }
}

ZB_DEVICE double pow2(int e) {
    // exact 2^e for the normal range; ldexp handles the rest
    if (e >= -1022 && e <= 1023) return __longlong_as_double((long long)(e + 1023) << 52);
    return ldexp(1.0, e);
}

// 2 KB after the barriers: per-tile column scale factors of the epilogue.
ZB_DEVICE uint8_t* smem_tail_scratch(uint8_t* smem) {
    return smem + kASlots * kAChunk + kBSlots * kBChunk + 256;
}
// Barrier among the four epilogue warps only (named barrier 1, 128 threads).
ZB_DEVICE void epilogue_bar_sync() { asm volatile("bar.sync 1, 128;\n" ::: "memory"); }
// The same barrier, returning the AND of every epilogue thread's `ok`: the
// four warps leave the tile loop together when any of them saw a wait fail
// (a warp that left alone would strand the others at the next barrier).
ZB_DEVICE bool epilogue_bar_and(bool ok) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, 128, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)ok)
        : "memory");
    return r != 0;
}

// Slot ring bookkeeping shared by the producer and the MMA issuer.
struct Ring {
    int slot = 0;
    uint32_t phase = 0;
    ZB_DEVICE void advance(int n) {
        if (++slot == n) {
            slot = 0;
            phase ^= 1;
        }
    }
};

// ------------------------------------------ Ozaki scheme II (CRT) tables
// Pairwise coprime moduli <= 256: residues are int8 in [-128, 127] and a
// modular product sums k products of magnitude <= 2^14 in INT32.
constexpr int kCrtModuli[kCrtMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233,
                                           229, 227, 223, 211, 199, 197, 193, 191};

struct CrtTable {
    int m[kCrtMaxModuli];
    float inv[kCrtMaxModuli];
    uint32_t wlo[kCrtMaxModuli], whi[kCrtMaxModuli];  // int8 x4: 2^(8t) mod m for t = 0..3 / 4..7
    int bias[kCrtMaxModuli];                          // 2^63 mod m
    int magic[kCrtMaxModuli];  // 0x4B400000 - bias: the dp4a sum reads as the FP32 number 1.5 2^23 + value
};

// Symmetric representative of r mod m: [-128, 127] for m = 256, |x| <= (m-1)/2 for odd m.
constexpr int sym_residue(long long r, int m) {
    long long x = r % m;
    if (x < 0) x += m;
    return (int)(x >= (m + 1) / 2 ? x - m : x);
}

constexpr CrtTable make_crt_table() {
    CrtTable t{};
    for (int l = 0; l < kCrtMaxModuli; ++l) {
        const int m = kCrtModuli[l];
        t.m[l] = m;
        t.inv[l] = 1.0f / (float)m;
        long long p = 1;  // 2^(8 b) mod m
        uint32_t lo = 0, hi = 0;
        for (int b = 0; b < 8; ++b) {
            const uint32_t byte = (uint32_t)(sym_residue(p, m) & 0xFF);
            if (b < 4)
                lo |= byte << (8 * b);
            else
                hi |= byte << (8 * (b - 4));
            p = (p * 256) % m;
        }
        t.wlo[l] = lo;
        t.whi[l] = hi;
        long long q = 1;
        for (int b = 0; b < 63; ++b) q = (q * 2) % m;
        t.bias[l] = sym_residue(q, m);
        // |sum_t byte_t w_t| <= 8 * 255 * 128 < 2^18: adding m * ceil((2^18 + 128) / m) keeps it >= 0
        t.magic[l] = 0x4B400000 - t.bias[l];
    }
    return t;
}

__constant__ CrtTable kCrt = make_crt_table();

// Exponent marker of a row of op(A) (column of op(B)) holding Inf or NaN: its
// digits / residues are zero, the emulated product leaves its entries of C
// alone and ozaki_nonfinite_patch computes them in IEEE FP64 afterwards.
constexpr int kNonFinite = -0x40000000;

// d = c + sum_i a.u8[i] * b.s8[i]
ZB_DEVICE int dp4a_us(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// v mod m, symmetric, for |v| < 2^31 - 2^21: the first FP32 quotient is
// within 2 of v / m, the second is exact, the result lies in [-m/2, m/2] and
// +128 (m = 256 only) folds to -128.
ZB_DEVICE int crt_reduce(int v, int m, float inv) {
    int q = __float2int_rn(__int2float_rn(v) * inv);
    v -= q * m;
    q = __float2int_rn(__int2float_rn(v) * inv);
    v -= q * m;
    return v > 127 ? v - m : v;
}

// 32 INT32 modular products of one TMEM lane -> 32 int8 residues (32 bytes of
// one row of a row-major residue plane).
ZB_DEVICE void residue_chunk(const uint32_t (&r)[32], int mod_idx, int8_t* dst) {
    uint32_t w[8];
    if (mod_idx == 0) {  // m = 256: the low byte of the two's-complement sum
#pragma unroll
        for (int q = 0; q < 8; ++q)
            w[q] = (r[4 * q] & 0xFFu) | ((r[4 * q + 1] & 0xFFu) << 8) | ((r[4 * q + 2] & 0xFFu) << 16) |
                   (r[4 * q + 3] << 24);
    } else {
        const int m = kCrt.m[mod_idx];
        const float inv = kCrt.inv[mod_idx];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            uint32_t x = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) x |= ((uint32_t)crt_reduce((int)r[4 * q + i], m, inv) & 0xFFu) << (8 * i);
            w[q] = x;
        }
    }
    // streaming stores: the residues are read once, by the reconstruction, and
    // should not displace the operand planes the other tiles still read from L2
    uint4* d = reinterpret_cast<uint4*>(dst);
    __stcs(d, make_uint4(w[0], w[1], w[2], w[3]));
    __stcs(d + 1, make_uint4(w[4], w[5], w[6], w[7]));
}

// Per-step flags of the job schedule, staged in shared memory once per CTA so
// the single MMA-issuing thread reads one byte per step instead of indexing
// the parameter space.
enum : uint8_t { SF_ACC1 = 1, SF_NEW_A = 2, SF_NEW_B = 4, SF_REL_A = 8, SF_REL_B = 16 };

struct Sched {
    uint8_t flags[kMaxSteps];
    uint8_t a[kMaxSteps];
    uint8_t b[kMaxSteps];
};

ZB_DEVICE void build_sched(const UmmaParams& P, Sched* s) {
    for (int j = 0; j < P.num_jobs; ++j) {
        const int f0 = P.job_first_step[j], n = P.job_num_steps[j];
        for (int q = 0; q < n; ++q) {
            const int st = f0 + q;
            uint8_t f = P.step_acc[st] ? SF_ACC1 : 0;
            if (q == 0 || P.step_a[st] != P.step_a[st - 1]) f |= SF_NEW_A;
            if (q == 0 || P.step_b[st] != P.step_b[st - 1]) f |= SF_NEW_B;
            if (q == n - 1 || P.step_a[st + 1] != P.step_a[st]) f |= SF_REL_A;
            if (q == n - 1 || P.step_b[st + 1] != P.step_b[st]) f |= SF_REL_B;
            s->flags[st] = f;
            s->a[st] = (uint8_t)P.step_a[st];
            s->b[st] = (uint8_t)P.step_b[st];
        }
    }
}

// MMA issue for one job over K chunks [c0, c1): 4 UMMAs (K = 4 x 32 bytes)
// per step, operand descriptors built once per slot and advanced by 32 bytes
// (+2 in the descriptor's 16-byte address units) per UMMA.
template <int ASLOTS, int BSLOTS, int ACHUNK, int BCHUNK, class Mma, class Commit>
ZB_DEVICE bool mma_job(const uint8_t* flags, int n_steps, int c0, int c1, Ring& ra, Ring& rb, uint64_t* fullA,
                       uint64_t* fullB, uint64_t* emptyA, uint64_t* emptyB, uint32_t sA0, uint32_t sB0,
                       uint32_t tmem_base, const WaitCtl& w, Mma mma, Commit commit) {
    uint32_t started = 0;
    uint64_t adesc = 0, bdesc = 0;
    int a_slot = 0, b_slot = 0;
    for (int kc = c0; kc < c1; ++kc) {
        for (int q = 0; q < n_steps; ++q) {
            const uint32_t f = flags[q];
            if (f & SF_NEW_A) {
                a_slot = ra.slot;
                if (!wait_phase(&fullA[a_slot], ra.phase, w, WAIT_MMA_FULL_A)) return false;
                ra.advance(ASLOTS);
                adesc = umma_desc_sw128(sA0 + a_slot * ACHUNK);
            }
            if (f & SF_NEW_B) {
                b_slot = rb.slot;
                if (!wait_phase(&fullB[b_slot], rb.phase, w, WAIT_MMA_FULL_B)) return false;
                rb.advance(BSLOTS);
                bdesc = umma_desc_sw128(sB0 + b_slot * BCHUNK);
            }
            const uint32_t acc_i = f & SF_ACC1;
            const uint32_t d = tmem_base + acc_i * kUN;
            mma(d, adesc, bdesc, (started >> acc_i) & 1u);
            mma(d, adesc + 2, bdesc + 2, 1u);
            mma(d, adesc + 4, bdesc + 4, 1u);
            mma(d, adesc + 6, bdesc + 6, 1u);
            started |= 1u << acc_i;
            if (f & SF_REL_A) commit(&emptyA[a_slot]);
            if (f & SF_REL_B) commit(&emptyB[b_slot]);
        }
    }
    return true;
}

template <int KIND, int EPI>
__global__ void __launch_bounds__(kThreads, 1)
umma_slice_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ UmmaParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + kASlots * kAChunk;
    uint64_t* fullA = reinterpret_cast<uint64_t*>(sB + kBSlots * kBChunk);
    uint64_t* emptyA = fullA + kASlots;
    uint64_t* fullB = emptyA + kASlots;
    uint64_t* emptyB = fullB + kBSlots;
    uint64_t* tfull = emptyB + kBSlots;  // [2]
    uint64_t* tempty = tfull + 2;        // [2]
    uint64_t* hold_bar = tempty + 2;     // test-only: nothing ever arrives on it
    uint64_t* drain_bar = hold_bar + 1;  // abort path: the MMA issuer's last commit
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    Sched* sched = reinterpret_cast<Sched*>(smem_tail_scratch(smem) + kUN * 8);
    const WaitCtl W{abort_flag, P.status, P.report, P.wait_ns};

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 32) build_sched(P, sched);
    if (threadIdx.x == 0) {
        for (int i = 0; i < kASlots; ++i) {
            mbar_init(&fullA[i], 1);
            mbar_init(&emptyA[i], 1);
        }
        for (int i = 0; i < kBSlots; ++i) {
            mbar_init(&fullB[i], 1);
            mbar_init(&emptyB[i], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);
        }
        mbar_init(hold_bar, 1);
        mbar_init(drain_bar, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        __syncwarp();  // lane 0 built the schedule; the allocation is warp-wide
        tmem_alloc(tmem_slot, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // launched during the tail of the residue / digit split that writes the planes
    grid_dependency_wait();
    const uint32_t tmem_base = *tmem_slot;
    const int elems_per_chunk = (KIND == KIND_I8) ? kChunkBytes : kChunkBytes / 2;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            Ring ra, rb;
            Issued ia, ib;
            bool ok = true;
            for (int tile = blockIdx.x; ok && tile < P.num_tiles; tile += gridDim.x) {
                int tm, tn;
                tile_coords(tile, P.tiles_m, P.tiles_n, tm, tn);
                for (int j = 0; ok && j < P.num_jobs; ++j)
                    for (int ks = 0; ok && ks < P.num_kseg; ++ks) {
                        const int c1 = min(P.k_chunks, (ks + 1) * P.kseg_chunks);
                        const int f0 = P.job_first_step[j], n_steps = P.job_num_steps[j];
                        for (int kc = ks * P.kseg_chunks; ok && kc < c1; ++kc) {
                            for (int q = 0; q < n_steps; ++q) {
                                const uint32_t f = sched->flags[f0 + q];
                                if (f & SF_NEW_A) {
                                    if (!(ok = wait_phase(&emptyA[ra.slot], ra.phase ^ 1, W, WAIT_PRODUCER_EMPTY_A)))
                                        break;
                                    mbar_arrive_expect_tx(&fullA[ra.slot], kAChunk);
                                    tma_load_2d(smem_u32(sA + ra.slot * kAChunk), &tmA, &fullA[ra.slot],
                                                kc * elems_per_chunk, sched->a[f0 + q] * P.m_pad + tm * kUM);
                                    ia.note(ra.slot, ra.phase);
                                    ra.advance(kASlots);
                                }
                                if (f & SF_NEW_B) {
                                    if (!(ok = wait_phase(&emptyB[rb.slot], rb.phase ^ 1, W, WAIT_PRODUCER_EMPTY_B)))
                                        break;
                                    mbar_arrive_expect_tx(&fullB[rb.slot], kBChunk);
                                    tma_load_2d(smem_u32(sB + rb.slot * kBChunk), &tmB, &fullB[rb.slot],
                                                kc * elems_per_chunk, sched->b[f0 + q] * P.n_pad + tn * kUN);
                                    ib.note(rb.slot, rb.phase);
                                    rb.advance(kBSlots);
                                }
                            }
                        }
                    }
            }
            if (ok) {
                // every issued copy was consumed by an MMA before the CTA retires
                for (int i = 0; i < kASlots; ++i) {
                    wait_phase(&emptyA[ra.slot], ra.phase ^ 1, W, 0);
                    ra.advance(kASlots);
                }
                for (int i = 0; i < kBSlots; ++i) {
                    wait_phase(&emptyB[rb.slot], rb.phase ^ 1, W, 0);
                    rb.advance(kBSlots);
                }
            } else {
                // aborted: let the bytes of every issued copy land before the CTA retires
                ia.drain(fullA, kASlots, P.wait_ns);
                ib.drain(fullB, kBSlots, P.wait_ns);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = (KIND == KIND_I8) ? umma_idesc(2, 1, kUM, kUN) : umma_idesc(1, 1, kUM, kUN);
            Ring ra, rb;
            uint32_t tphase = 0;  // bit b: phase parity of accumulator buffer b
            bool ok = !P.hold || wait_phase(hold_bar, 0, W, WAIT_MMA_HOLD);
            int inst = 0;
            for (int tile = blockIdx.x; ok && tile < P.num_tiles; tile += gridDim.x)
                for (int j = 0; ok && j < P.num_jobs; ++j)
                    for (int ks = 0; ok && ks < P.num_kseg; ++ks) {
                        // the job's accumulators must have been drained by the epilogue
                        // EPI_F32 (one accumulator per tile) alternates the two TMEM buffers
                        // so a tile's epilogue overlaps the next tile's products
                        const int b = (EPI == EPI_RESIDUE) ? P.job_buf[j] : (EPI == EPI_F32 ? (inst & 1) : 0);
                        ++inst;
                        if (!(ok = wait_phase(&tempty[b], ((tphase >> b) & 1u) ^ 1u, W, WAIT_MMA_TEMPTY))) break;
                        tphase ^= 1u << b;
                        tc_fence_after();
                        const int c0 = ks * P.kseg_chunks, c1 = min(P.k_chunks, (ks + 1) * P.kseg_chunks);
                        auto mma = [idesc](uint32_t d, uint64_t ad, uint64_t bd, uint32_t acc) {
                            if (KIND == KIND_I8)
                                umma_i8(d, ad, bd, idesc, acc);
                            else
                                umma_f16(d, ad, bd, idesc, acc);
                        };
                        auto commit = [](uint64_t* bar) { umma_commit(bar); };
                        ok = mma_job<kASlots, kBSlots, kAChunk, kBChunk>(
                            sched->flags + P.job_first_step[j], P.job_num_steps[j], c0, c1, ra, rb, fullA, fullB,
                            emptyA, emptyB, smem_u32(sA), smem_u32(sB), tmem_base + (EPI == EPI_F32 ? b * kUN : 0), W, mma,
                            commit);
                        if (ok) umma_commit(&tfull[b]);
                    }
            if (!ok) {
                // aborted: the MMAs already issued read shared memory and write
                // TMEM; wait for them before either is released
                umma_commit(drain_bar);
                drain_phase(drain_bar, 0, P.wait_ns);
            }
        }
    } else {
        // ---------------------------------------------- epilogue warps
        const int quarter = warp & 3;  // TMEM lane quarter this warp may access
        const int row_in_tile = quarter * 32 + lane;
        const int et = threadIdx.x - 64;  // 0..127 among the epilogue threads
        const uint32_t lane_addr = tmem_base + ((uint32_t)(quarter * 32) << 16);
        double* colscale = reinterpret_cast<double*>(smem_tail_scratch(smem));  // kUN doubles
        uint32_t tphase = 0;  // bit b: phase parity of accumulator buffer b
        int inst = 0;  // accumulator instances, in the MMA issuer's order
        bool ok = true;
        for (int tile = blockIdx.x; tile < P.num_tiles; tile += gridDim.x) {
            int tm, tn;
            tile_coords(tile, P.tiles_m, P.tiles_n, tm, tn);
            const int row = tm * kUM + row_in_tile;
            bool row_ok = row < P.m;
            int er = 0;
            if (EPI == EPI_OZAKI_F64) {
                // all four warps leave together; the previous tile's readers are done
                if (!epilogue_bar_and(ok)) break;
                if (row_ok) er = P.row_exp[row];
                row_ok = row_ok && er != kNonFinite;  // left to the non-finite patch
                // 2^{f_j} of this tile's columns, staged once per tile (-1: a
                // column of op(B) holding Inf / NaN, left to the patch)
                for (int c = et; c < kUN; c += 128) {
                    const int col = tn * kUN + c;
                    const int ec = (col < P.n) ? P.col_exp[col] : 0;
                    colscale[c] = (col < P.n) ? (ec == kNonFinite ? -1.0 : pow2(ec)) : 0.0;
                }
                epilogue_bar_sync();
            } else if (!ok) {
                break;
            }
            bool first = true;
            for (int j = 0; ok && j < P.num_jobs; ++j)
                for (int ks = 0; ok && ks < P.num_kseg; ++ks) {
                    const int b = (EPI == EPI_RESIDUE) ? P.job_buf[j] : (EPI == EPI_F32 ? (inst & 1) : 0);
                    ++inst;
                    if (!(ok = wait_phase(&tfull[b], (tphase >> b) & 1u, W, WAIT_EPILOGUE_TFULL))) break;
                    tphase ^= 1u << b;
                    tc_fence_after();
                    if (EPI == EPI_RESIDUE) {
                        // one modulus per job: accumulator b -> int8 residues, row-major plane
                        int8_t* dst = P.residues + (long)P.job_shift[j][0] * P.res_plane + (long)row * P.n_pad +
                                      (long)tn * kUN;
#pragma unroll 1
                        for (int ch = 0; ch < kUN / 32; ++ch) {
                            uint32_t r0[32];
                            tmem_ld_32x32b_x32(lane_addr + b * kUN + ch * 32, r0);
                            tmem_ld_wait();
                            residue_chunk(r0, P.job_shift[j][0], dst + ch * 32);
                        }
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&tempty[b]);
                        continue;
                    }
                    const bool two = P.job_groups[j] == 2;
                    // accumulator 1 holds group g_a - 1, worth 2^7 times accumulator 0:
                    // D0 + 128 D1 is exact in int64 and converts exactly to FP64.
                    const double s0 = (EPI == EPI_OZAKI_F64) ? pow2(er - P.job_shift[j][0]) * P.alpha : 1.0;
#pragma unroll 1
                    for (int ch = 0; ch < kUN / 32; ++ch) {
                        uint32_t r0[32], r1[32];
                        tmem_ld_32x32b_x32(lane_addr + (EPI == EPI_F32 ? b * kUN : 0) + ch * 32, r0);
                        if (two) tmem_ld_32x32b_x32(lane_addr + kUN + ch * 32, r1);
                        tmem_ld_wait();
                        const int col0 = tn * kUN + ch * 32;
                        if (!row_ok) continue;
                        const bool full_chunk = col0 + 32 <= P.n;
                        // Issue all loads of C before any store so their
                        // round trips overlap.
                        if (EPI == EPI_OZAKI_F64) {
                            double* cb = static_cast<double*>(P.c) + (long)col0 * P.ldc + row;
                            double cin[32];
                            const bool need_c = !first || P.beta != 0.0;
                            if (need_c) {
#pragma unroll
                                for (int c = 0; c < 32; ++c)
                                    cin[c] = (full_chunk || col0 + c < P.n) ? __ldcg(cb + (long)c * P.ldc) : 0.0;
                            }
                            const double* cs = colscale + ch * 32;
#pragma unroll
                            for (int c = 0; c < 32; ++c) {
                                long long d = (int)r0[c];
                                if (two) d += (long long)(int)r1[c] << 7;
                                const double v = (double)d * s0 * cs[c];
                                const double out = !need_c ? v : (first ? fma(P.beta, cin[c], v) : cin[c] + v);
                                if ((full_chunk || col0 + c < P.n) && cs[c] >= 0.0) __stcg(cb + (long)c * P.ldc, out);
                            }
                        } else {
                            float* cb = static_cast<float*>(P.c) + (long)col0 * P.ldc + row;
                            float cin[32];
                            const bool need_c = !first || P.beta_f != 0.0f;
                            if (need_c) {
#pragma unroll
                                for (int c = 0; c < 32; ++c)
                                    cin[c] = (full_chunk || col0 + c < P.n) ? __ldcg(cb + (long)c * P.ldc) : 0.0f;
                            }
#pragma unroll
                            for (int c = 0; c < 32; ++c) {
                                const float v = P.alpha_f * __uint_as_float(r0[c]);
                                const float out = !need_c ? v : (first ? fmaf(P.beta_f, cin[c], v) : cin[c] + v);
                                if (full_chunk || col0 + c < P.n) __stcg(cb + (long)c * P.ldc, out);
                            }
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&tempty[b]);
                    first = false;
                }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem_base, 512);
}

// ------------------------------------------------- 2-CTA (cta_group::2)
// The same schedule on a CTA pair: one M = 256 x N = 256 UMMA per K step,
// issued by the even CTA.  CTA r loads A rows [256 tm + 128 r, +128) and B
// rows [256 tn + 128 r, +128) into its own shared memory (the tensor cores
// read both halves), and its TMEM receives C rows [256 tm + 128 r, +128) x 256.
// Per SM this halves the B bytes of every chunk.  TMA completion bytes of both
// CTAs are counted on the even CTA's "full" barriers; the MMA commits arrive on
// the "empty" / "tfull" barriers of both CTAs (tcgen05.commit multicast); the
// odd CTA's epilogue arrives on the even CTA's "tempty" barrier remotely.
constexpr int kSlots2 = 6;                      // A and B rings, 128 x 128 B each
constexpr int kChunk2 = 128 * kChunkBytes;      // 16 KB
constexpr size_t kSmemBytes2 = 1024 + 2 * kSlots2 * kChunk2 + 512 + kUN * 8 + 3 * kMaxSteps;
// CRT residue products on the CTA pair: every step needs a fresh A and B
// chunk, so a slot holds 256 bytes of K of both operands (two 128-byte swizzle
// atoms each: A0 A1 B0 B1, 16 KB per atom and CTA) behind one full / empty
// barrier pair, and a step issues 8 UMMAs per barrier round trip.
constexpr int kCrtAtom = 128 * kChunkBytes;  // 16 KB
constexpr int kCrtSlot = 4 * kCrtAtom;       // 64 KB
constexpr int kCrtSlots = (2 * kSlots2 * kChunk2) / kCrtSlot;  // 3
static_assert(kCrtSlots >= 2, "CRT ring");

// A CTA of the pair cannot observe its own copies land (their bytes are
// counted on the even CTA's barriers); after an abort it waits this long for
// them (a TMA copy of one slot takes a few microseconds).
constexpr unsigned long long kPeerCopyGraceNs = 200000;

template <int KIND, int EPI>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
umma_slice_gemm_2cta(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const __grid_constant__ UmmaParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + kSlots2 * kChunk2;
    uint64_t* fullA = reinterpret_cast<uint64_t*>(sB + kSlots2 * kChunk2);
    uint64_t* emptyA = fullA + kSlots2;
    uint64_t* fullB = emptyA + kSlots2;
    uint64_t* emptyB = fullB + kSlots2;
    uint64_t* tfull = emptyB + kSlots2;  // [2]
    uint64_t* tempty = tfull + 2;        // [2]
    uint64_t* hold_bar = tempty + 2;     // test-only: nothing ever arrives on it
    uint64_t* drain_bar = hold_bar + 1;  // abort path: the MMA issuer's last commit (even CTA)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    double* colscale = reinterpret_cast<double*>(sB + kSlots2 * kChunk2 + 512);
    Sched* sched = reinterpret_cast<Sched*>(sB + kSlots2 * kChunk2 + 512 + kUN * 8);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 32) build_sched(P, sched);
    const uint32_t rank = cluster_ctarank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    // an abort raised in either CTA is raised in both
    const WaitCtl W{abort_flag, P.status, P.report, P.wait_ns,
                    mapa_shared(smem_u32(const_cast<int*>(abort_flag)), rank ^ 1u)};
    if (threadIdx.x == 0) {
        for (int i = 0; i < kSlots2; ++i) {
            mbar_init(&fullA[i], 1);
            mbar_init(&emptyA[i], 1);
            mbar_init(&fullB[i], 1);
            mbar_init(&emptyB[i], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 8);  // 4 epilogue warps in each CTA of the pair
        }
        mbar_init(hold_bar, 1);
        mbar_init(drain_bar, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        __syncwarp();  // lane 0 built the schedule; the allocation is warp-wide
        tmem_alloc_2sm(tmem_slot, 512);
        tmem_relinquish_2sm();
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // the peer's barriers (and abort flag) exist before any remote access
    tc_fence_after();
    // launched during the tail of the residue / digit split that writes the planes
    grid_dependency_wait();
    const uint32_t tmem_base = *tmem_slot;
    const int elems_per_chunk = (KIND == KIND_I8) ? kChunkBytes : kChunkBytes / 2;

    if (warp == 0 && EPI == EPI_RESIDUE) {
        // ------------------------------------- TMA producer, CRT residue products
        if (lane == 0) {
            Ring rs;
            Issued is;
            bool ok = true;
            const int steps = P.k_chunks / 2;  // 256-byte K steps (K padded to 256)
            // modulus-major over one flat sequence q = (modulus, tile), dealt
            // round-robin to the pairs: every pair gets the same number of
            // items (within one), so the running pairs stay on neighbouring
            // tiles of one modulus and share its planes in L2 (a per-modulus
            // deal of 13 or 14 tiles let the pairs drift moduli apart)
            for (int q = pair; ok && q < P.num_jobs * P.num_tiles; q += npairs) {
                const int j = q / P.num_tiles, tile = q - j * P.num_tiles;
                int tm, tn;
                crt_job_tile(P.tri, tile, P.tiles_m, P.tiles_n, P.band_rows, tm, tn);
                const int arow = tm * 256 + rank * 128, brow = tn * kUN + rank * 128;
                const int l = P.job_shift[j][0];
                for (int ks = 0; ks < steps; ++ks) {
                    if (!(ok = wait_phase(&emptyA[rs.slot], rs.phase ^ 1, W, WAIT_PRODUCER_EMPTY_A))) break;
                    const uint32_t base = smem_u32(smem) + rs.slot * kCrtSlot;
                    const uint32_t bar = smem_u32(&fullA[rs.slot]) & 0xFEFFFFFFu;
                    if (leader) mbar_arrive_expect_tx(&fullA[rs.slot], 2 * kCrtSlot);
                    const int x = ks * 2 * kChunkBytes;
                    tma_load_2d_2sm(base, &tmA, bar, x, l * P.m_pad + arow);
                    tma_load_2d_2sm(base + kCrtAtom, &tmA, bar, x + kChunkBytes, l * P.m_pad + arow);
                    tma_load_2d_2sm(base + 2 * kCrtAtom, &tmB, bar, x, l * P.n_pad + brow);
                    tma_load_2d_2sm(base + 3 * kCrtAtom, &tmB, bar, x + kChunkBytes, l * P.n_pad + brow);
                    is.note(rs.slot, rs.phase);
                    rs.advance(kCrtSlots);
                }
            }
            if (ok) {
                for (int i = 0; i < kCrtSlots; ++i) {
                    wait_phase(&emptyA[rs.slot], rs.phase ^ 1, W, 0);
                    rs.advance(kCrtSlots);
                }
            } else if (leader) {
                is.drain(fullA, kCrtSlots, P.wait_ns);  // both CTAs' bytes of every issued slot
            } else {
                spin_ns(kPeerCopyGraceNs);
            }
        }
    } else if (warp == 1 && EPI == EPI_RESIDUE) {
        // ------------------------------------ MMA issuer (even CTA), CRT products
        if (lane == 0 && leader) {
            const uint32_t idesc = umma_idesc(2, 1, 256, kUN);
            Ring rs;
            uint32_t tphase = 0;
            bool ok = !P.hold || wait_phase(hold_bar, 0, W, WAIT_MMA_HOLD);
            const int steps = P.k_chunks / 2;
            int inst = 0;  // job instances alternate between the two accumulators
            for (int q = pair; ok && q < P.num_jobs * P.num_tiles; q += npairs) {
                const int b = inst++ & 1;
                if (!(ok = wait_phase(&tempty[b], ((tphase >> b) & 1u) ^ 1u, W, WAIT_MMA_TEMPTY))) break;
                tphase ^= 1u << b;
                tc_fence_after();
                const uint32_t d = tmem_base + b * kUN;
                for (int ks = 0; ks < steps; ++ks) {
                    if (!(ok = wait_phase(&fullA[rs.slot], rs.phase, W, WAIT_MMA_FULL_A))) break;
                    const uint32_t base = smem_u32(smem) + rs.slot * kCrtSlot;
                    const uint64_t a0 = umma_desc_sw128(base), a1 = umma_desc_sw128(base + kCrtAtom);
                    const uint64_t b0 = umma_desc_sw128(base + 2 * kCrtAtom);
                    const uint64_t b1 = umma_desc_sw128(base + 3 * kCrtAtom);
                    umma_i8_2sm(d, a0, b0, idesc, ks > 0 ? 1u : 0u);
                    umma_i8_2sm(d, a0 + 2, b0 + 2, idesc, 1u);
                    umma_i8_2sm(d, a0 + 4, b0 + 4, idesc, 1u);
                    umma_i8_2sm(d, a0 + 6, b0 + 6, idesc, 1u);
                    umma_i8_2sm(d, a1, b1, idesc, 1u);
                    umma_i8_2sm(d, a1 + 2, b1 + 2, idesc, 1u);
                    umma_i8_2sm(d, a1 + 4, b1 + 4, idesc, 1u);
                    umma_i8_2sm(d, a1 + 6, b1 + 6, idesc, 1u);
                    umma_commit_2sm(&emptyA[rs.slot], 0x3);
                    rs.advance(kCrtSlots);
                }
                if (ok) umma_commit_2sm(&tfull[b], 0x3);
            }
            if (!ok) {
                // aborted: wait for the MMAs already issued before TMEM and the ring are released
                umma_commit_2sm(drain_bar, 0x1);
                drain_phase(drain_bar, 0, P.wait_ns);
            }
        }
    } else if (warp == 0) {
        // ------------------------------------------------ TMA producer (both CTAs)
        if (lane == 0) {
            Ring ra, rb;
            Issued ia, ib;
            bool ok = true;
            for (int tile = pair; ok && tile < P.num_tiles; tile += npairs) {
                int tm, tn;
                tile_coords(tile, P.tiles_m, P.tiles_n, tm, tn);
                const int arow = tm * 256 + rank * 128, brow = tn * kUN + rank * 128;
                for (int j = 0; ok && j < P.num_jobs; ++j)
                    for (int ks = 0; ok && ks < P.num_kseg; ++ks) {
                        const int c1 = min(P.k_chunks, (ks + 1) * P.kseg_chunks);
                        const int f0 = P.job_first_step[j], n_steps = P.job_num_steps[j];
                        for (int kc = ks * P.kseg_chunks; ok && kc < c1; ++kc) {
                            for (int q = 0; q < n_steps; ++q) {
                                const uint32_t f = sched->flags[f0 + q];
                                if (f & SF_NEW_A) {
                                    if (!(ok = wait_phase(&emptyA[ra.slot], ra.phase ^ 1, W, WAIT_PRODUCER_EMPTY_A)))
                                        break;
                                    if (leader) mbar_arrive_expect_tx(&fullA[ra.slot], 2 * kChunk2);
                                    tma_load_2d_2sm(smem_u32(sA + ra.slot * kChunk2), &tmA,
                                                    smem_u32(&fullA[ra.slot]) & 0xFEFFFFFFu, kc * elems_per_chunk,
                                                    sched->a[f0 + q] * P.m_pad + arow);
                                    ia.note(ra.slot, ra.phase);
                                    ra.advance(kSlots2);
                                }
                                if (f & SF_NEW_B) {
                                    if (!(ok = wait_phase(&emptyB[rb.slot], rb.phase ^ 1, W, WAIT_PRODUCER_EMPTY_B)))
                                        break;
                                    if (leader) mbar_arrive_expect_tx(&fullB[rb.slot], 2 * kChunk2);
                                    tma_load_2d_2sm(smem_u32(sB + rb.slot * kChunk2), &tmB,
                                                    smem_u32(&fullB[rb.slot]) & 0xFEFFFFFFu, kc * elems_per_chunk,
                                                    sched->b[f0 + q] * P.n_pad + brow);
                                    ib.note(rb.slot, rb.phase);
                                    rb.advance(kSlots2);
                                }
                            }
                        }
                    }
            }
            if (ok) {
                for (int i = 0; i < kSlots2; ++i) {
                    wait_phase(&emptyA[ra.slot], ra.phase ^ 1, W, 0);
                    ra.advance(kSlots2);
                    wait_phase(&emptyB[rb.slot], rb.phase ^ 1, W, 0);
                    rb.advance(kSlots2);
                }
            } else if (leader) {
                ia.drain(fullA, kSlots2, P.wait_ns);
                ib.drain(fullB, kSlots2, P.wait_ns);
            } else {
                spin_ns(kPeerCopyGraceNs);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------- MMA issuer (even CTA)
        if (lane == 0 && leader) {
            const uint32_t idesc = (KIND == KIND_I8) ? umma_idesc(2, 1, 256, kUN) : umma_idesc(1, 1, 256, kUN);
            Ring ra, rb;
            uint32_t tphase = 0;  // bit b: phase parity of accumulator buffer b
            bool ok = !P.hold || wait_phase(hold_bar, 0, W, WAIT_MMA_HOLD);
            int inst = 0;
            for (int tile = pair; ok && tile < P.num_tiles; tile += npairs)
                for (int j = 0; ok && j < P.num_jobs; ++j)
                    for (int ks = 0; ok && ks < P.num_kseg; ++ks) {
                        // EPI_F32 (one accumulator per tile) alternates the two TMEM buffers
                        // so a tile's epilogue overlaps the next tile's products
                        const int b = (EPI == EPI_RESIDUE) ? P.job_buf[j] : (EPI == EPI_F32 ? (inst & 1) : 0);
                        ++inst;
                        if (!(ok = wait_phase(&tempty[b], ((tphase >> b) & 1u) ^ 1u, W, WAIT_MMA_TEMPTY))) break;
                        tphase ^= 1u << b;
                        tc_fence_after();
                        const int c0 = ks * P.kseg_chunks, c1 = min(P.k_chunks, (ks + 1) * P.kseg_chunks);
                        auto mma = [idesc](uint32_t d, uint64_t ad, uint64_t bd, uint32_t acc) {
                            if (KIND == KIND_I8)
                                umma_i8_2sm(d, ad, bd, idesc, acc);
                            else
                                umma_f16_2sm(d, ad, bd, idesc, acc);
                        };
                        auto commit = [](uint64_t* bar) { umma_commit_2sm(bar, 0x3); };
                        ok = mma_job<kSlots2, kSlots2, kChunk2, kChunk2>(
                            sched->flags + P.job_first_step[j], P.job_num_steps[j], c0, c1, ra, rb, fullA, fullB,
                            emptyA, emptyB, smem_u32(sA), smem_u32(sB), tmem_base + (EPI == EPI_F32 ? b * kUN : 0), W, mma,
                            commit);
                        if (ok) umma_commit_2sm(&tfull[b], 0x3);
                    }
            if (!ok) {
                umma_commit_2sm(drain_bar, 0x1);
                drain_phase(drain_bar, 0, P.wait_ns);
            }
        }
    } else {
        // ---------------------------------------------- epilogue warps (both CTAs)
        const int quarter = warp & 3;
        const int row_in_tile = rank * 128 + quarter * 32 + lane;
        const int et = threadIdx.x - 64;
        const uint32_t lane_addr = tmem_base + ((uint32_t)(quarter * 32) << 16);
        const uint32_t tempty_cta0 = mapa_shared(smem_u32(&tempty[0]), 0);  // buffer b: + 8 b
        uint32_t tphase = 0;  // bit b: phase parity of accumulator buffer b
        int inst = 0;  // accumulator instances, in the MMA issuer's order
        bool ok = true;
        if (EPI == EPI_RESIDUE) {
            // modulus-major, in the order of the MMA issuer
            int inst = 0;
            for (int q = pair; ok && q < P.num_jobs * P.num_tiles; q += npairs) {
                const int j = q / P.num_tiles, tile = q - j * P.num_tiles;
                int tm, tn;
                crt_job_tile(P.tri, tile, P.tiles_m, P.tiles_n, P.band_rows, tm, tn);
                const int b = inst++ & 1;
                if (!(ok = wait_phase(&tfull[b], (tphase >> b) & 1u, W, WAIT_EPILOGUE_TFULL))) break;
                tphase ^= 1u << b;
                tc_fence_after();
                const int row = tm * 256 + row_in_tile;
                int8_t* dst = P.residues + (long)P.job_shift[j][0] * P.res_plane + (long)row * P.n_pad +
                              (long)tn * kUN;
#pragma unroll 1
                for (int ch = 0; ch < kUN / 32; ++ch) {
                    uint32_t r0[32];
                    tmem_ld_32x32b_x32(lane_addr + b * kUN + ch * 32, r0);
                    tmem_ld_wait();
                    residue_chunk(r0, P.job_shift[j][0], dst + ch * 32);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(tempty_cta0 + 8u * b);
            }
        }
        for (int tile = pair; EPI != EPI_RESIDUE && tile < P.num_tiles; tile += npairs) {
            int tm, tn;
            tile_coords(tile, P.tiles_m, P.tiles_n, tm, tn);
            const int row = tm * 256 + row_in_tile;
            bool row_ok = row < P.m;
            int er = 0;
            if (EPI == EPI_OZAKI_F64) {
                if (!epilogue_bar_and(ok)) break;  // all four warps leave together
                if (row_ok) er = P.row_exp[row];
                row_ok = row_ok && er != kNonFinite;  // left to the non-finite patch
                for (int c = et; c < kUN; c += 128) {
                    const int col = tn * kUN + c;
                    const int ec = (col < P.n) ? P.col_exp[col] : 0;
                    colscale[c] = (col < P.n) ? (ec == kNonFinite ? -1.0 : pow2(ec)) : 0.0;
                }
                epilogue_bar_sync();
            } else if (!ok) {
                break;
            }
            bool first = true;
            for (int j = 0; ok && j < P.num_jobs; ++j)
                for (int ks = 0; ok && ks < P.num_kseg; ++ks) {
                    const int b = (EPI == EPI_RESIDUE) ? P.job_buf[j] : (EPI == EPI_F32 ? (inst & 1) : 0);
                    ++inst;
                    if (!(ok = wait_phase(&tfull[b], (tphase >> b) & 1u, W, WAIT_EPILOGUE_TFULL))) break;
                    tphase ^= 1u << b;
                    tc_fence_after();
                    const bool two = P.job_groups[j] == 2;
                    const double s0 = (EPI == EPI_OZAKI_F64) ? pow2(er - P.job_shift[j][0]) * P.alpha : 1.0;
#pragma unroll 1
                    for (int ch = 0; ch < kUN / 32; ++ch) {
                        uint32_t r0[32], r1[32];
                        tmem_ld_32x32b_x32(lane_addr + (EPI == EPI_F32 ? b * kUN : 0) + ch * 32, r0);
                        if (two) tmem_ld_32x32b_x32(lane_addr + kUN + ch * 32, r1);
                        tmem_ld_wait();
                        const int col0 = tn * kUN + ch * 32;
                        if (!row_ok) continue;
                        const bool full_chunk = col0 + 32 <= P.n;
                        if (EPI == EPI_OZAKI_F64) {
                            double* cb = static_cast<double*>(P.c) + (long)col0 * P.ldc + row;
                            double cin[32];
                            const bool need_c = !first || P.beta != 0.0;
                            if (need_c) {
#pragma unroll
                                for (int c = 0; c < 32; ++c)
                                    cin[c] = (full_chunk || col0 + c < P.n) ? __ldcg(cb + (long)c * P.ldc) : 0.0;
                            }
                            const double* cs = colscale + ch * 32;
#pragma unroll
                            for (int c = 0; c < 32; ++c) {
                                long long d = (int)r0[c];
                                if (two) d += (long long)(int)r1[c] << 7;
                                const double v = (double)d * s0 * cs[c];
                                const double out = !need_c ? v : (first ? fma(P.beta, cin[c], v) : cin[c] + v);
                                if ((full_chunk || col0 + c < P.n) && cs[c] >= 0.0) __stcg(cb + (long)c * P.ldc, out);
                            }
                        } else {
                            float* cb = static_cast<float*>(P.c) + (long)col0 * P.ldc + row;
                            float cin[32];
                            const bool need_c = !first || P.beta_f != 0.0f;
                            if (need_c) {
#pragma unroll
                                for (int c = 0; c < 32; ++c)
                                    cin[c] = (full_chunk || col0 + c < P.n) ? __ldcg(cb + (long)c * P.ldc) : 0.0f;
                            }
#pragma unroll
                            for (int c = 0; c < 32; ++c) {
                                const float v = P.alpha_f * __uint_as_float(r0[c]);
                                const float out = !need_c ? v : (first ? fmaf(P.beta_f, cin[c], v) : cin[c] + v);
                                if (full_chunk || col0 + c < P.n) __stcg(cb + (long)c * P.ldc, out);
                            }
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive_cluster(tempty_cta0 + 8u * b);
                    first = false;
                }
        }
    }

    tc_fence_before();
    __syncthreads();
    cluster_sync();  // no CTA of the pair leaves while the other's MMAs or loads may touch it
    tc_fence_after();
    if (warp == 1) tmem_dealloc_2sm(tmem_base, 512);
}

// ------------------------------------------------------------- splitting
// View of a matrix X (rows r, cols c): element at base[r * rs + c * cs];
// exactly one of rs / cs is 1.
template <typename T>
struct ViewT {
    const T* base;
    long rs, cs;
    int rows, cols;
};
using View = ViewT<double>;
using ViewF = ViewT<float>;

// |x| bit patterns at or above this one are Inf or NaN.
constexpr unsigned long long kInfBits = 0x7FF0000000000000ull;

// Append row r to the list of rows holding Inf / NaN (rows of op(A) or
// columns of op(B)); the non-finite patch reads the list after the product.
ZB_DEVICE void note_nonfinite(int r, int* count, int* list) { list[atomicAdd(count, 1)] = r; }

// Row maxima of |X| as FP64 bit patterns (non-negative doubles order like
// unsigned integers; NaN patterns sort above +Inf and so propagate).
// Also accumulates the row sums of |x| (used by the automatic slice count and
// the CRT row scale).  T = float reads FP32 operands, widened exactly.
template <typename T>
__global__ void ozaki_absmax(ViewT<T> X, unsigned long long* __restrict__ maxbits, double* __restrict__ sums) {
    grid_dependency_wait();  // may be launched during the tail of the kernel before it
    if (X.rs == 1) {
        const int r = blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= X.rows) return;
        const int c0 = blockIdx.y * 64, c1 = min(X.cols, c0 + 64);
        unsigned long long mx = 0;
        double sm = 0.0;
        for (int c = c0; c < c1; ++c) {
            const double a = fabs((double)X.base[r + (long)c * X.cs]);
            const unsigned long long v = (unsigned long long)__double_as_longlong(a);
            mx = v > mx ? v : mx;
            sm += a;
        }
        if (mx) atomicMax(&maxbits[r], mx);
        if (sm != 0.0) atomicAdd(&sums[r], sm);
    } else {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int r = blockIdx.x * (blockDim.x / 32) + warp;
        if (r >= X.rows) return;
        const int c0 = blockIdx.y * 1024, c1 = min(X.cols, c0 + 1024);
        unsigned long long mx = 0;
        double sm = 0.0;
        for (int c = c0 + lane; c < c1; c += 32) {
            const double a = fabs((double)X.base[(long)r * X.rs + c]);
            const unsigned long long v = (unsigned long long)__double_as_longlong(a);
            mx = v > mx ? v : mx;
            sm += a;
        }
        for (int o = 16; o; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, mx, o);
            mx = w > mx ? w : mx;
            sm += __shfl_xor_sync(0xffffffffu, sm, o);
        }
        if (lane == 0 && mx) atomicMax(&maxbits[r], mx);
        if (lane == 0 && sm != 0.0) atomicAdd(&sums[r], sm);
    }
}

// Largest "spread" over rows: e_r - log2(mean_c |x_rc|), the number of bits
// between a row's scaling exponent and its typical magnitude.  The digits of
// a typical entry start this many bits below the top of the first slice.
__global__ void ozaki_spread(const unsigned long long* __restrict__ maxbits, const double* __restrict__ sums,
                             int rows, int cols, float* __restrict__ out) {
    float best = 0.f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
        if (maxbits[r] == 0 || maxbits[r] >= kInfBits || !(sums[r] > 0.0)) continue;  // zero or non-finite row
        int e;
        frexp(__longlong_as_double((long long)maxbits[r]), &e);
        const float sp = (float)(e - log2(sums[r] / cols));
        best = sp > best ? sp : best;
    }
    for (int o = 16; o; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    __shared__ float part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmaxf(b, part[w]);
        *out = b;
    }
}

// Exponent e with max * 2^-e in [0.5, 1): the frexp exponent of the maximum
// (kNonFinite for a row holding Inf or NaN).
ZB_DEVICE int row_exponent(unsigned long long bits) {
    if (bits == 0) return 0;
    if (bits >= kInfBits) return kNonFinite;
    int e;
    frexp(__longlong_as_double((long long)bits), &e);
    return e;
}

// Swizzled [32][128] double tile: conflict-free both for 32 consecutive rows
// of one column and for 16 consecutive columns of two adjacent rows.
ZB_DEVICE int swz(int r, int c) {
    const int h = ((r & 1) << 3) | ((r >> 1) & 7);
    return r * 128 + (c ^ ((h ^ (c >> 4)) & 15));
}

// Each block: 32 rows x 128 columns of X -> s int8 digit planes
// (plane t: rows_pad x cols_pad bytes, K-major) and the row exponents.
__global__ void __launch_bounds__(256)
ozaki_split(View X, const unsigned long long* __restrict__ maxbits, int slices, int rows_pad, int cols_pad,
            int8_t* __restrict__ planes, int* __restrict__ exps, int* __restrict__ nf_count, int* __restrict__ nf_list) {
    __shared__ double tile[32 * 128];
    __shared__ int sexp[32];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 128;
    const int t = threadIdx.x;
    if (t < 32) {
        const int r = r0 + t;
        const int e = (r < X.rows) ? row_exponent(maxbits[r]) : 0;
        sexp[t] = e;
        if (blockIdx.x == 0 && r < rows_pad) exps[r] = e;
        if (blockIdx.x == 0 && r < X.rows && e == kNonFinite) note_nonfinite(r, nf_count, nf_list);
    }
    // load (coalesced along the contiguous dimension of X)
#pragma unroll 4
    for (int it = 0; it < 16; ++it) {
        const int idx = it * 256 + t;
        int r, c;
        if (X.rs == 1) {
            r = idx & 31;
            c = idx >> 5;
        } else {
            r = idx >> 7;
            c = idx & 127;
        }
        const int gr = r0 + r, gc = c0 + c;
        double v = 0.0;
        if (gr < X.rows && gc < X.cols) v = (double)X.base[(long)gr * X.rs + (long)gc * X.cs];
        tile[swz(r, c)] = v;
    }
    __syncthreads();
    // digits: thread -> row t / 8, 16 consecutive columns
    const int r = t >> 3, q = t & 7;
    // a row holding Inf / NaN gets zero digits (its entries of C are patched)
    const double sc = sexp[r] == kNonFinite ? 0.0 : ldexp(1.0, -sexp[r]);
    double y[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) y[i] = sc == 0.0 ? 0.0 : tile[swz(r, q * 16 + i)] * sc;
    const long plane = (long)rows_pad * cols_pad;
    int8_t* out = planes + (long)(r0 + r) * cols_pad + c0 + q * 16;
    for (int s = 0; s < slices; ++s) {
        uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const double z = y[i] * 128.0;
            const double d = trunc(z);
            y[i] = z - d;
            w[i >> 2] |= ((uint32_t)(int)d & 0xFFu) << (8 * (i & 3));
        }
        if (r0 + r < rows_pad) *reinterpret_cast<uint4*>(out + s * plane) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// ---------------------------------------------- CRT residues of operands
// Row scale of the CRT scheme: 2^{a_r} with ||2^{a_r} x_r||_2 <= 2^P, from the
// Hoelder bound ||x_r||_2 <= sqrt(max_r * sum_r) <= max_r * sqrt(min(sum_r / max_r, k)).
ZB_DEVICE int crt_row_exponent(unsigned long long maxbits, double sum, int k, int P) {
    if (maxbits == 0) return 0;
    const double mx = __longlong_as_double((long long)maxbits);
    if (!(mx <= 1.7976931348623157e308)) return kNonFinite;  // Inf or NaN in the row
    int e1, e2;
    const double f1 = frexp(mx, &e1);  // mx = f1 2^e1, f1 in [0.5, 1)
    const double ratio = fmin(sum / mx, (double)k);
    frexp(f1 * sqrt(fmax(ratio, 1.0)) * (1.0 + 0x1p-20), &e2);  // < 2^e2
    return P - (e1 + e2);
}

// Two FP32 lanes per instruction (sm_100 packed FP32): d = a * b + c, d = a + b.
ZB_DEVICE uint64_t ffma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;\n" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
ZB_DEVICE uint64_t fadd2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;\n" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
ZB_DEVICE uint64_t pack2(uint32_t lo, uint32_t hi) { return (uint64_t)hi << 32 | lo; }
ZB_DEVICE uint64_t pack2f(float lo, float hi) { return pack2(__float_as_uint(lo), __float_as_uint(hi)); }

// Each block: 32 rows x 128 columns of X -> `nmod` int8 residue planes
// (plane l: rows_pad x cols_pad bytes, K-major) of round(2^{a_r} x) and the
// row exponents a_r.  The integer (|.| <= 2^P <= 2^62) is biased by 2^63 so
// that its eight bytes are unsigned digits; residue = dp4a(bytes, 2^{8t} mod m)
// - (2^63 mod m), then one exact FP32 reduction.  T = float: FP32 operands,
// widened exactly to FP64 on load.
template <typename T>
__global__ void __launch_bounds__(256)
ozaki_crt_split(ViewT<T> X, const unsigned long long* __restrict__ maxbits, const double* __restrict__ sums, int P,
                int nmod, int rows_pad, int cols_pad, int8_t* __restrict__ planes, int* __restrict__ exps,
                int* __restrict__ nf_count, int* __restrict__ nf_list) {
    __shared__ double tile[32 * 128];
    __shared__ int sexp[32];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 128;
    const int t = threadIdx.x;
    grid_dependency_wait();  // launched during the tail of the statistics pass
    if (t < 32) {
        const int r = r0 + t;
        const int e = (r < X.rows) ? crt_row_exponent(maxbits[r], sums[r], X.cols, P) : 0;
        sexp[t] = e;
        if (blockIdx.x == 0 && r < rows_pad) exps[r] = e;
        if (blockIdx.x == 0 && r < X.rows && e == kNonFinite) note_nonfinite(r, nf_count, nf_list);
    }
#pragma unroll 4
    for (int it = 0; it < 16; ++it) {
        const int idx = it * 256 + t;
        int r, c;
        if (X.rs == 1) {
            r = idx & 31;
            c = idx >> 5;
        } else {
            r = idx >> 7;
            c = idx & 127;
        }
        const int gr = r0 + r, gc = c0 + c;
        double v = 0.0;
        if (gr < X.rows && gc < X.cols) v = (double)X.base[(long)gr * X.rs + (long)gc * X.cs];
        tile[swz(r, c)] = v;
    }
    __syncthreads();
    const int r = t >> 3, q = t & 7;
    if (r0 + r >= rows_pad) return;
    const int a = sexp[r];
    const bool finite = a != kNonFinite;
    // 2^a by one exact multiplication when both 2^a and the products stay normal
    const bool plain = a >= -960 && a <= 960;
    const double sc = plain ? pow2(a) : 0.0;
    uint32_t lo[16], hi[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const double x = tile[swz(r, q * 16 + i)];
        const long long v = !finite ? 0LL : __double2ll_rn(plain ? x * sc : ldexp(x, a));
        const unsigned long long u = (unsigned long long)v ^ (1ull << 63);
        lo[i] = (uint32_t)u;
        hi[i] = (uint32_t)(u >> 32);
    }
    const long plane = (long)rows_pad * cols_pad;
    int8_t* out = planes + (long)(r0 + r) * cols_pad + c0 + q * 16;
    // modulus 256: the low byte of the integer
    {
        uint32_t w[4];
#pragma unroll
        for (int g = 0; g < 4; ++g)
            w[g] = (lo[4 * g] & 0xFFu) | ((lo[4 * g + 1] & 0xFFu) << 8) | ((lo[4 * g + 2] & 0xFFu) << 16) |
                   (lo[4 * g + 3] << 24);
        *reinterpret_cast<uint4*>(out) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    const uint64_t kMagic2 = pack2f(12582912.0f, 12582912.0f), kNegMagic2 = pack2f(-12582912.0f, -12582912.0f);
    for (int l = 1; l < nmod; ++l) {
        const float m = (float)kCrt.m[l], inv = kCrt.inv[l];
        const uint64_t m2 = pack2f(-m, -m), inv2 = pack2f(inv, inv);
        const uint32_t wl = kCrt.wlo[l], wh = kCrt.whi[l];
        const int c0 = kCrt.magic[l];
        uint32_t w[4];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            // value v = sum_t byte_t (2^8t mod m) - (2^63 mod m), |v| < 2^18; the dp4a
            // result is the bit pattern of the float f = 1.5 2^23 + v, so x = v exactly;
            // q = round(v / m) by the 1.5 2^23 shift; f - q m = 1.5 2^23 + r is exact
            // with |r| <= (m - 1) / 2 and carries r in the low byte of its pattern.  The
            // FP32 steps run on two entries per instruction (f32x2).
            uint32_t d[4], rb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) d[i] = (uint32_t)dp4a_us(lo[4 * g + i], wl, dp4a_us(hi[4 * g + i], wh, c0));
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint64_t f = pack2(d[2 * h], d[2 * h + 1]);
                const uint64_t q = fadd2(ffma2(fadd2(f, kNegMagic2), inv2, kMagic2), kNegMagic2);
                const uint64_t r = ffma2(q, m2, f);
                rb[2 * h] = (uint32_t)r;
                rb[2 * h + 1] = (uint32_t)(r >> 32);
            }
            w[g] = __byte_perm(__byte_perm(rb[0], rb[1], 0x0040), __byte_perm(rb[2], rb[3], 0x0040), 0x5410);
        }
        *reinterpret_cast<uint4*>(out + l * plane) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// CRT weights w_l = M_l (M_l^-1 mod m_l) mod M and M = prod m_l (< 2^127 for
// 16 moduli).  The weights are held as 16 balanced base-256 digits d_{l,z} in
// [-128, 127], packed as the B operand of an int8 m16n8k16 MMA: wb[h][t][g]
// holds d_{4t+i, 8h+g} in byte i (moduli 4t .. 4t+3, digit 8h + g).  M itself
// is kept as eight balanced 16-bit limbs for the reduction S - q M.
constexpr int kCrtLimbs = 8;
struct CrtCombine {
    int nmod;
    uint32_t wb[2][4][8];
    int M[kCrtLimbs];
    double M_d, inv_M;
};

constexpr double pow2_const(int e) {
    double x = 1.0;
    for (int i = 0; i < e; ++i) x *= 2.0;
    return x;
}

// Exact int32 -> FP64 without the conversion unit: the bits 0x43300000:(v ^ 2^31)
// encode 2^52 + 2^31 + v.
ZB_DEVICE double i2d(int v) {
    return __hiloint2double(0x43300000, v ^ 0x80000000) - 4503601774854144.0;  // 2^52 + 2^31
}

// D (16 x 8, s32) = A (16 x 16, s8, row) B (16 x 8, s8, col): lane (g, t) holds
// a0 = A[g][4t .. 4t+3], a1 = A[g+8][4t .. 4t+3], b = B[4t .. 4t+3][g] and
// receives D[g][2t, 2t+1] (d0, d1), D[g+8][2t, 2t+1] (d2, d3).
ZB_DEVICE void imma_16x8x16(int (&d)[4], uint32_t a0, uint32_t a1, uint32_t b) {
    asm("mma.sync.aligned.m16n8k16.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%7,%7,%7,%7};\n"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3])
        : "r"(a0), "r"(a1), "r"(b), "r"(0));
}

constexpr int kLimbStride = 9;  // words per element in the limb buffer: conflict-free stores and loads

// C = alpha 2^{-(a_i + b_j)} CRT(r_0..r_{n-1}) + beta C on a 16 x 128 tile of
// row-major residue planes.  Warp w takes rows w and w + 8 in two 64-column
// segments each.  The digit sums S_z = sum_l r_l d_{l,z} of 64 elements x 16
// digits are a product (64 x 16 residues) (16 x 16 digits) on the int8 tensor
// pipe: MMA tile u holds the columns 4x + u (x = 0..15) of the segment, so the
// four bytes at columns 4g .. 4g+3 of moduli 4t .. 4t+3 (one 4-byte load per
// modulus) byte-transpose into the A fragments of all four tiles.  Lane (g, t)
// then holds the 16-bit limbs S_{2y} + 256 S_{2y+1} (y = t, 4 + t) of eight
// elements; a per-warp shared buffer regroups them so that lane L owns all
// eight limbs of columns L and 32 + L (|limb| < 2^27, exact in int32).
// q = round(S / M) from an FP64 estimate (|C_bar| <= M / 4 keeps S / M near an
// integer); C_bar = S - q M is carried to balanced 16-bit limbs and rounded to
// FP64 from the top limb down.  The scaled results pass through shared memory
// so that C (column-major) is written 128 bytes per column.  T = float: the
// FP64 value alpha x + beta C is rounded once to FP32.
template <int NMOD, typename T>
__global__ void __launch_bounds__(256)
ozaki_crt_combine(const int8_t* __restrict__ res, long plane, int res_ld, int m, int n, const int* __restrict__ expa,
                  const int* __restrict__ expb, double alpha, double beta, T* __restrict__ C, long ldc,
                  const __grid_constant__ CrtCombine K, const int* __restrict__ status, int tri) {
    // every modulus is >= 191 > 2^7.5, so log2 M >= 7.5 NMOD
    constexpr int Z0 = (15 * NMOD - 78) > 0 ? (15 * NMOD - 78) / 32 : 0;
    constexpr double kScaleZ0 = pow2_const(16 * Z0);
    grid_dependency_wait();  // launched during the tail of the products that write the residues
    // The modular products did not all complete (a bounded wait ran out): C stays as it was.
    if (*status) return;
    // triangle mode: blocks with no entry of the stored triangle (their residues were not computed)
    if ((tri == 1 && (int)blockIdx.x * 16 > (int)blockIdx.y * 128 + 127) ||
        (tri == 2 && (int)blockIdx.x * 16 + 15 < (int)blockIdx.y * 128))
        return;
    __shared__ double ct[16][129];
    __shared__ int lb[8][64 * kLimbStride];
    __shared__ int sexa[16], sexb[128];  // row / column exponents (kNonFinite: Inf / NaN in the row / column)
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, g = lane >> 2, q4 = lane & 3;
    const int i0 = blockIdx.x * 16, j0 = blockIdx.y * 128;
    if (t < 128) sexb[t] = expb[j0 + t];  // < n_pad: the planes are padded to 256 columns
    if (t < 16) sexa[t] = expa[i0 + t];   // < m_pad: the planes are padded to 128 rows
    const uint32_t b_lo = K.wb[0][q4][g], b_hi = K.wb[1][q4][g];
    int* my = lb[warp];
    __syncthreads();
#pragma unroll 1
    for (int unit = 0; unit < 4; ++unit) {
        const int rl = warp + 8 * (unit >> 1), seg = unit & 1, gi = i0 + rl;
        const int8_t* rp = res + (long)gi * res_ld + j0 + seg * 64 + 4 * g;
        uint32_t v[2][4];
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int l = 4 * q4 + i;
                v[e2][i] = l < NMOD ? __ldcs(reinterpret_cast<const uint32_t*>(rp + l * plane + 32 * e2)) : 0u;
            }
        // a[e2][u]: residues of moduli 4t .. 4t+3 of column 4g + 32 e2 + u
        uint32_t a[2][4];
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            const uint32_t t0 = __byte_perm(v[e2][0], v[e2][1], 0x5140), t1 = __byte_perm(v[e2][2], v[e2][3], 0x5140);
            const uint32_t t2 = __byte_perm(v[e2][0], v[e2][1], 0x7362), t3 = __byte_perm(v[e2][2], v[e2][3], 0x7362);
            a[e2][0] = __byte_perm(t0, t1, 0x5410);
            a[e2][1] = __byte_perm(t0, t1, 0x7632);
            a[e2][2] = __byte_perm(t2, t3, 0x5410);
            a[e2][3] = __byte_perm(t2, t3, 0x7632);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            int dl[4], dh[4];
            imma_16x8x16(dl, a[0][u], a[1][u], b_lo);  // digits 2t, 2t+1
            imma_16x8x16(dh, a[0][u], a[1][u], b_hi);  // digits 8 + 2t, 9 + 2t
            const int e0 = 4 * g + u, e1 = 32 + 4 * g + u;
            my[e0 * kLimbStride + q4] = dl[0] + 256 * dl[1];
            my[e0 * kLimbStride + 4 + q4] = dh[0] + 256 * dh[1];
            my[e1 * kLimbStride + q4] = dl[2] + 256 * dl[3];
            my[e1 * kLimbStride + 4 + q4] = dh[2] + 256 * dh[3];
        }
        __syncwarp();
        const int ea = sexa[rl];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int e = lane + 32 * s;
            int c[kCrtLimbs];
#pragma unroll
            for (int z = 0; z < kCrtLimbs; ++z) c[z] = my[e * kLimbStride + z];
            // limbs below Z0 add less than 2^(16 Z0 + 27) <= M 2^-12 to S, so the
            // upper limbs place S / M within 2^-12 of its value
            double sd = i2d(c[kCrtLimbs - 1]);
#pragma unroll
            for (int z = kCrtLimbs - 2; z >= Z0; --z) sd = fma(sd, 65536.0, i2d(c[z]));
            sd *= kScaleZ0;
            const int qq = __double2int_rn(sd * K.inv_M);
#pragma unroll
            for (int z = 0; z < kCrtLimbs; ++z) c[z] -= qq * K.M[z];
#pragma unroll
            for (int z = 0; z < kCrtLimbs - 1; ++z) {
                const int carry = (c[z] + 32768) >> 16;
                c[z] -= carry << 16;
                c[z + 1] += carry;
            }
            double x = i2d(c[kCrtLimbs - 1]);
#pragma unroll
            for (int z = kCrtLimbs - 2; z >= 0; --z) x = fma(x, 65536.0, i2d(c[z]));
            const int sc = -(ea + sexb[seg * 64 + e]);
            ct[rl][seg * 64 + e] = alpha * (sc >= -1022 && sc <= 1023 ? x * pow2(sc) : ldexp(x, sc));
        }
        __syncwarp();  // the buffer is refilled by the next unit
    }
    __syncthreads();
    // column-major write: 16 consecutive rows (128 bytes) of one column per half-warp
    const int r = t & 15;
    const int gi = i0 + r;
    if (gi >= m || sexa[r] == kNonFinite) return;  // rows holding Inf / NaN: left to the non-finite patch
#pragma unroll 4
    for (int cc = t >> 4; cc < 128; cc += 16) {
        const int gj = j0 + cc;
        if (gj >= n) break;
        if (sexb[cc] == kNonFinite) continue;
        T* cp = C + (long)gj * ldc + gi;
        double out = ct[r][cc];
        if (beta != 0.0) out = fma(beta, (double)*cp, out);
        *cp = (T)out;
    }
}

template <typename T>
using CombineFn = void (*)(const int8_t*, long, int, int, int, const int*, const int*, double, double, T*, long,
                           CrtCombine, const int*, int);
template <int N, typename T>
constexpr CombineFn<T> combine_at(int nmod) {
    if constexpr (N == 1)
        return &ozaki_crt_combine<1, T>;
    else
        return nmod == N ? &ozaki_crt_combine<N, T> : combine_at<N - 1, T>(nmod);
}

// IEEE semantics for rows of op(A) / columns of op(B) that hold Inf or NaN.
// Their integer digits / residues are zero and the emulated product leaves
// their entries of C untouched; this kernel then computes exactly those
// entries as plain FP64 dot products, C = alpha * sum_p A_ip B_pj (+ beta C
// when beta != 0), the reference's loop (gemm.zig:1422-1429).  Every such
// entry is Inf or NaN, and which one does not depend on the summation order.
// Work items are 64 x 64 output tiles: rows listed in list_a x all columns,
// then all rows (except listed ones) x columns listed in list_b; a persistent
// grid reads the two counts, so with no Inf / NaN in the operands every CTA
// returns at once.  A warp whose listed rows / columns lie past the count
// skips its arithmetic.
constexpr int kPatchTile = 64, kPatchK = 16;

template <typename T>
__global__ void __launch_bounds__(256)
ozaki_nonfinite_patch(ViewT<T> va, ViewT<T> vb, int m, int n, int k, double alpha, double beta, T* __restrict__ C,
                      long ldc, const int* __restrict__ cnt_a, const int* __restrict__ list_a,
                      const int* __restrict__ cnt_b, const int* __restrict__ list_b, const int* __restrict__ expa,
                      const int* __restrict__ status) {
    grid_dependency_wait();  // launched during the tail of the reconstruction that writes C
    if (*status) return;  // the product did not complete: C stays as it was
    const int na = *cnt_a, nb = *cnt_b;
    if (na == 0 && nb == 0) return;
    __shared__ double Gs[kPatchK][kPatchTile + 1];  // [p][listed row / column]
    __shared__ double Ds[kPatchK][kPatchTile + 1];  // [p][dense row / column]
    const int t = threadIdx.x, warp = t >> 5;
    const int ty = t >> 4, tx = t & 15;  // outputs: listed ty*4 + u, dense tx + 16 v
    const long items_a = (long)((na + kPatchTile - 1) / kPatchTile) * ((n + kPatchTile - 1) / kPatchTile);
    const long items_b = (long)((nb + kPatchTile - 1) / kPatchTile) * ((m + kPatchTile - 1) / kPatchTile);
    for (long item = blockIdx.x; item < items_a + items_b; item += gridDim.x) {
        // listed side G (rows of op(A), or columns of op(B) = rows of op(B)^T), dense side D
        const bool rows = item < items_a;
        const long it = rows ? item : item - items_a;
        const int dense_ext = rows ? n : m;
        const int dense_tiles = (dense_ext + kPatchTile - 1) / kPatchTile;
        const int g0 = (int)(it / dense_tiles) * kPatchTile, d0 = (int)(it % dense_tiles) * kPatchTile;
        const int gcount = min(kPatchTile, (rows ? na : nb) - g0);
        const int* list = rows ? list_a : list_b;
        const ViewT<T>& G = rows ? va : vb;
        const ViewT<T>& D = rows ? vb : va;
        const bool warp_busy = warp * 8 < gcount;
        double acc[4][4] = {};
        for (int p0 = 0; p0 < k; p0 += kPatchK) {
            __syncthreads();  // the previous slice's readers are done
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int e = t + 256 * q;
                // contiguous index fastest in global memory
                int gr, gp;
                if (G.cs == 1) { gp = e % kPatchK; gr = e / kPatchK; } else { gr = e % kPatchTile; gp = e / kPatchTile; }
                double v = 0.0;
                if (gr < gcount && p0 + gp < k) v = (double)G.base[(long)list[g0 + gr] * G.rs + (long)(p0 + gp) * G.cs];
                Gs[gp][gr] = v;
                int dr, dp;
                if (D.cs == 1) { dp = e % kPatchK; dr = e / kPatchK; } else { dr = e % kPatchTile; dp = e / kPatchTile; }
                double w = 0.0;
                if (d0 + dr < dense_ext && p0 + dp < k) w = (double)D.base[(long)(d0 + dr) * D.rs + (long)(p0 + dp) * D.cs];
                Ds[dp][dr] = w;
            }
            __syncthreads();
            if (warp_busy) {
#pragma unroll 4
                for (int p = 0; p < kPatchK; ++p) {
                    double gv[4], dv[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) gv[u] = Gs[p][ty * 4 + u];
#pragma unroll
                    for (int v = 0; v < 4; ++v) dv[v] = Ds[p][tx + 16 * v];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) acc[u][v] = fma(gv[u], dv[v], acc[u][v]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int g = ty * 4 + u;
            if (g >= gcount) continue;
            const int listed = list[g0 + g];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int d = d0 + tx + 16 * v;
                if (d >= dense_ext) continue;
                const int i = rows ? listed : d, j = rows ? d : listed;
                if (!rows && expa[i] == kNonFinite) continue;  // the row pass wrote it
                T* cp = C + (long)j * ldc + i;
                double out = alpha * acc[u][v];
                if (beta != 0.0) out = out + beta * (double)*cp;
                *cp = (T)out;
            }
        }
    }
}

// 3xBF16 split of a float matrix view into hi / lo planes (bf16, K-major).
__global__ void __launch_bounds__(256)
bf16_split(ViewF X, int rows_pad, int cols_pad, __nv_bfloat16* __restrict__ planes) {
    __shared__ float tile[32][129];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 128;
    const int t = threadIdx.x;
#pragma unroll 4
    for (int it = 0; it < 16; ++it) {
        const int idx = it * 256 + t;
        int r, c;
        if (X.rs == 1) {
            r = idx & 31;
            c = idx >> 5;
        } else {
            r = idx >> 7;
            c = idx & 127;
        }
        const int gr = r0 + r, gc = c0 + c;
        float v = 0.f;
        if (gr < X.rows && gc < X.cols) v = X.base[(long)gr * X.rs + (long)gc * X.cs];
        tile[r][c] = v;
    }
    __syncthreads();
    const int r = t >> 3, q = t & 7;
    if (r0 + r >= rows_pad) return;
    const long plane = (long)rows_pad * cols_pad;
    __nv_bfloat16 hi[16], lo[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const float x = tile[r][q * 16 + i];
        hi[i] = __float2bfloat16_rn(x);
        lo[i] = __float2bfloat16_rn(x - __bfloat162float(hi[i]));
    }
    __nv_bfloat16* o = planes + (long)(r0 + r) * cols_pad + c0 + q * 16;
    *reinterpret_cast<uint4*>(o) = *reinterpret_cast<uint4*>(hi);
    *reinterpret_cast<uint4*>(o + 8) = *reinterpret_cast<uint4*>(hi + 8);
    *reinterpret_cast<uint4*>(o + plane) = *reinterpret_cast<uint4*>(lo);
    *reinterpret_cast<uint4*>(o + plane + 8) = *reinterpret_cast<uint4*>(lo + 8);
}

// ------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
}

// 2-D K-major digit tensor: inner dim = K (cols_pad elements), outer = planes * rows_pad rows.
cudaError_t make_map(CUtensorMap* map, const void* base, CUtensorMapDataType dt, int elem_bytes, long cols_pad,
                     long total_rows, int box_rows) {
    auto enc = get_encode();
    if (!enc) return cudaErrorNotSupported;
    cuuint64_t dims[2] = {(cuuint64_t)cols_pad, (cuuint64_t)total_rows};
    cuuint64_t strides[1] = {(cuuint64_t)(cols_pad * elem_bytes)};
    cuuint32_t box[2] = {(cuuint32_t)(kChunkBytes / elem_bytes), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

inline long round_up(long x, long m) { return (x + m - 1) / m * m; }

// Workspace layout: the small statistics block first, the digit planes after it.
// The statistics of op(A) come first and those of op(B) (with the status word)
// after them, so that a call reusing op(A) (a_ready) clears one range.
struct Layout {
    long maxa_off, suma_off, cnta_off, maxb_off, sumb_off, cntb_off, status_off, spread_off, b_clear_end;
    long expa_off, expb_off, lista_off, listb_off, stats_end;
    long a_planes_off, b_planes_off, res_off, total;
};

Layout ozaki_layout(const OzakiPlan& p) {
    Layout L{};
    long off = 0;
    auto take = [&](long bytes) {
        long o = off;
        off = round_up(off + bytes, 256);
        return o;
    };
    L.maxa_off = take((long)p.m_pad * 8);
    L.suma_off = take((long)p.m_pad * 8);
    L.cnta_off = take(16);
    L.maxb_off = take((long)p.n_pad * 8);
    L.sumb_off = take((long)p.n_pad * 8);
    L.cntb_off = take(16);
    L.status_off = take(64);
    L.spread_off = take(16);
    L.b_clear_end = off;
    L.expa_off = take((long)p.m_pad * 4);
    L.expb_off = take((long)p.n_pad * 4);
    L.lista_off = take((long)p.m_pad * 4);
    L.listb_off = take((long)p.n_pad * 4);
    L.stats_end = off;
    off = round_up(off, 1024);
    const int s = p.scheme == OZAKI_CRT ? p.moduli : (p.slices > 0 ? p.slices : kOzakiAutoMaxSlices);
    L.a_planes_off = take((long)s * p.m_pad * p.k_pad);
    L.b_planes_off = take((long)s * p.n_pad * p.k_pad);
    L.res_off = take(p.scheme == OZAKI_CRT ? (long)p.moduli * p.m_pad * p.n_pad : 0);
    L.total = off;
    return L;
}

int sm_count_cached() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// Per-device report word of bounded waits that ran out (0: none since the host
// last read it).  Host code reaches it through its device address, looked up
// once per device with that device current.
__device__ int g_wait_report;

constexpr int kMaxReportDevices = 64;
struct ReportSlot {
    std::once_flag once;
    int* ptr = nullptr;
    cudaError_t err = cudaSuccess;
};
ReportSlot g_report_slots[kMaxReportDevices];
// Set once any product kernel has been launched in this process (until then
// there is nothing to read, and reading would load this file's module).
std::atomic<bool> g_products_launched{false};

cudaError_t report_word(int** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxReportDevices) return cudaErrorInvalidDevice;
    ReportSlot& r = g_report_slots[dev];
    std::call_once(r.once, [&r] {
        void* q = nullptr;
        r.err = cudaGetSymbolAddress(&q, g_wait_report);
        r.ptr = static_cast<int*>(q);
    });
    *out = r.ptr;
    return r.err;
}

// Time limit of every mbarrier wait: generous for any legitimate wait (a job's
// products take microseconds, a context switch milliseconds); the test hold
// uses 1 ms so that the whole abort path runs in a few milliseconds.
constexpr unsigned long long kWaitLimitNs = 4000000000ull;
constexpr unsigned long long kHoldWaitLimitNs = 1000000ull;

cudaError_t set_wait_params(UmmaParams& P, bool hold) {
    cudaError_t e = report_word(&P.report);
    if (e != cudaSuccess) return e;
    P.hold = hold ? 1 : 0;
    P.wait_ns = hold ? kHoldWaitLimitNs : kWaitLimitNs;
    g_products_launched.store(true);
    return cudaSuccess;
}

// dependent: the kernel before it in the stream is one of this library's
// kernels (not a copy or memset), so the launch may overlap its tail.
template <int KIND, int EPI>
cudaError_t launch_umma(const CUtensorMap& ma, const CUtensorMap& mb, const UmmaParams& P, cudaStream_t st,
                        bool dependent = true) {
    auto kern = umma_slice_gemm<KIND, EPI>;
    cudaError_t e = ensure_dynamic_smem(kern, (int)kSmemBytes);
    if (e != cudaSuccess) return e;
    const int grid = P.num_tiles < sm_count_cached() ? P.num_tiles : sm_count_cached();
    prof_begin(st);
    if (dependent)
        e = launch_dependent(kern, dim3(grid), dim3(kThreads), kSmemBytes, st, ma, mb, P);
    else
        kern<<<grid, kThreads, kSmemBytes, st>>>(ma, mb, P);
    count_launch();
    prof_end(st);
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <int KIND, int EPI>
cudaError_t launch_umma_2cta(const CUtensorMap& ma, const CUtensorMap& mb, const UmmaParams& P, cudaStream_t st,
                             bool dependent = true) {
    auto kern = umma_slice_gemm_2cta<KIND, EPI>;
    cudaError_t e = ensure_dynamic_smem(kern, (int)kSmemBytes2);
    if (e != cudaSuccess) return e;
    // CRT residues deal independent (modulus, tile) items to the pairs, so a
    // product with fewer tiles than pairs still fills the GPU; the slice
    // epilogues keep every job of a tile on one pair
    const long items = EPI == EPI_RESIDUE ? (long)P.num_jobs * P.num_tiles : P.num_tiles;
    const int pairs = (int)std::min<long>(items, sm_count_cached() / 2);
    prof_begin(st);
    if (dependent)
        e = launch_dependent(kern, dim3(2 * pairs), dim3(kThreads), kSmemBytes2, st, ma, mb, P);
    else
        kern<<<2 * pairs, kThreads, kSmemBytes2, st>>>(ma, mb, P);
    count_launch();
    prof_end(st);
    return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace

// Largest K (in 128-byte chunks) whose INT32 group sums cannot overflow:
// pairs_per_group * K * 127^2 < 2^31.
static int max_kseg_chunks(int slices) {
    const long limit = (2147483647L / (long)(slices * 127 * 127)) / kChunkBytes;
    return limit < 1 ? 1 : (int)limit;
}

// The CTA-pair kernel is used from 256 rows up (ZYNUM_GPU_UMMA_2CTA=0 turns it off).
static bool use_cta_pair(int m) {
    static const bool enabled = [] {
        const char* v = std::getenv("ZYNUM_GPU_UMMA_2CTA");
        return !(v && v[0] == '0');
    }();
    return enabled && m >= 256;
}

// Automatic method choice from call times fitted to measured B200 runs (FP64
// through dgemm_device, 16 moduli, beta 1; shapes 256^3 .. 8192^3, 1536^3 and
// 3072^3, N = 512 and K = 512 panels).  Emulated: the 16 modular products at
// an effective 5.0 POPS, 7.0 ps per operand element (statistics and residues),
// 25.9 ps per C element (residue epilogue and reconstruction), 38.4 us of
// launches and per-kernel latency; relative error of the fit within 13 %.
// Native: 32 TFLOP/s plus 15 us.  Ozaki is taken below
// 0.9 x the native time; K beyond one CRT segment falls back to the slice
// scheme, which needs larger products still.
bool ozaki_preferred_scaled(int m, int n, int k, double native_fraction, double ozaki_fraction, double extra_bytes) {
    const double mnk2 = 2.0 * m * n * (double)k;
    const double native_s = native_fraction * mnk2 / 32e12 + 15e-6;
    const double ozaki_s = ozaki_fraction * (16.0 * mnk2 / 5.0e15 + 25.9e-12 * m * (double)n) +
                           7.0e-12 * ((double)m * k + (double)k * n) + extra_bytes / 6e12 + 38.4e-6;
    return k <= kCrtMaxK ? ozaki_s < 0.9 * native_s : native_fraction * mnk2 >= 2e12;
}

bool ozaki_preferred(int m, int n, int k) { return ozaki_preferred_scaled(m, n, k, 1.0, 1.0, 0.0); }

int ozaki_auto_slices(float spread_a, float spread_b) {
    // Truncating a row of A after s 7-bit digits leaves |dA_ik| < 2^(e_i - 7s)
    // with 2^e_i the row maximum; the spread is log2(row max / mean |A_ik|).
    // The error of the emulated product is then about
    //   2^-7s (2^spread_a + 2^spread_b) sum_k |A_ik| |B_kj|,
    // against about 2^-53 sum_k |A_ik| |B_kj| (with a data-dependent constant)
    // for native FP64, so s = ceil((52 + log2(2^sa + 2^sb)) / 7).  Checked at
    // 8192^3 on U[-1,1] * 10^U[-phi,phi] data for phi in {0, 2, 4, 8}: the
    // emulated max relative error is 4x (phi 0) to 30x (phi 4) below native.
    const float lead = fmaxf(spread_a, spread_b);
    const float both = lead + log2f(1.0f + exp2f(fminf(spread_a, spread_b) - lead));
    int s = (int)ceilf((52.0f + both) / 7.0f);
    if (s < 6) s = 6;
    if (s > kOzakiAutoMaxSlices) s = kOzakiAutoMaxSlices;
    return s;
}

namespace {
std::atomic<int> g_last_slices{0};
}
int ozaki_last_slices() { return g_last_slices.load(); }

OzakiPlan plan_ozaki(int m, int n, int k, int slices, int scheme, int moduli) {
    OzakiPlan p;
    if (slices > kOzakiMaxSlices) slices = kOzakiMaxSlices;
    if (slices < 0) slices = 0;
    const bool crt_ok = k <= kCrtMaxK;
    if (scheme == OZAKI_AUTO)
        scheme = (slices > 0 || !crt_ok) ? OZAKI_SLICES : OZAKI_CRT;
    else if (scheme == OZAKI_CRT && !crt_ok)
        scheme = OZAKI_SLICES;
    p.scheme = scheme == OZAKI_CRT ? OZAKI_CRT : OZAKI_SLICES;
    if (p.scheme == OZAKI_CRT) p.moduli = (moduli >= 2 && moduli <= kCrtMaxModuli) ? moduli : kCrtDefaultModuli;
    p.slices = slices;  // 0: chosen from the data at run time
    p.pair = use_cta_pair(m);
    p.m_pad = (int)round_up(m, p.pair ? 2 * kUM : kUM);
    p.n_pad = (int)round_up(n, kUN);
    // CRT: K in 256-byte steps on the CTA pair
    p.k_pad = (int)round_up(k, p.scheme == OZAKI_CRT ? 2 * kChunkBytes : kChunkBytes);
    return p;
}

size_t ozaki_workspace_bytes(const OzakiPlan& p) { return (size_t)ozaki_layout(p).total; }

namespace {
// Host constants of the CRT scheme for the first n moduli (exact in 128-bit
// integers: M < 2^127 for n <= 16) and the scaling bits P with 2^(2P) <= M / 4.
struct CrtHost {
    CrtCombine K;
    int P;
};

const CrtHost& crt_host(int nmod) {
    static CrtHost table[kCrtMaxModuli + 1];
    static std::once_flag once;
    std::call_once(once, [] {
        // balanced 16-bit limbs: x = sum_z out[z] 2^(16 z), out[z] in [-2^15, 2^15) (top limb: the rest)
        auto limbs = [](unsigned __int128 x, int* out) {
            long long L[kCrtLimbs];
            for (int z = 0; z < kCrtLimbs; ++z) L[z] = (long long)((x >> (16 * z)) & 0xFFFFu);
            for (int z = 0; z < kCrtLimbs - 1; ++z)
                if (L[z] >= (1LL << 15)) {
                    L[z] -= (1LL << 16);
                    L[z + 1] += 1;
                }
            for (int z = 0; z < kCrtLimbs; ++z) out[z] = (int)L[z];
        };
        // balanced base-256 digits: x = sum_z out[z] 256^z, out[z] in [-128, 128) (x < 2^126: the top one is small)
        auto digits = [](unsigned __int128 x, int* out) {
            long long D[16];
            for (int z = 0; z < 16; ++z) D[z] = (long long)((x >> (8 * z)) & 0xFFu);
            for (int z = 0; z < 15; ++z)
                if (D[z] >= 128) {
                    D[z] -= 256;
                    D[z + 1] += 1;
                }
            for (int z = 0; z < 16; ++z) out[z] = (int)D[z];
        };
        for (int n = 1; n <= kCrtMaxModuli; ++n) {
            unsigned __int128 M = 1;
            for (int l = 0; l < n; ++l) M *= (unsigned)kCrtModuli[l];
            CrtHost& h = table[n];
            h.K = CrtCombine{};
            h.K.nmod = n;
            int d[kCrtMaxModuli][16] = {};  // base-256 digits; moduli beyond n keep zero weights
            for (int l = 0; l < n; ++l) {
                const unsigned ml = (unsigned)kCrtModuli[l];
                const unsigned __int128 Ml = M / ml;
                const unsigned r = (unsigned)(Ml % ml);
                unsigned y = 1;
                for (unsigned c = 1; c < ml; ++c)
                    if ((r * c) % ml == 1) {
                        y = c;
                        break;
                    }
                digits(Ml * y % M, d[l]);
            }
            for (int hh = 0; hh < 2; ++hh)
                for (int t = 0; t < 4; ++t)
                    for (int g = 0; g < 8; ++g) {
                        uint32_t word = 0;
                        for (int i = 0; i < 4; ++i) word |= (uint32_t)(uint8_t)(int8_t)d[4 * t + i][8 * hh + g] << (8 * i);
                        h.K.wb[hh][t][g] = word;
                    }
            limbs(M, h.K.M);
            h.K.M_d = (double)M;
            h.K.inv_M = 1.0 / h.K.M_d;
            h.P = (int)std::floor((std::log2((double)M) - 2.0) / 2.0);
            if (h.P > 62) h.P = 62;  // the scaled integers stay inside int64
        }
    });
    return table[nmod];
}

std::atomic<int> g_last_moduli{0};

// Rows of op(A) / columns of op(B) holding Inf or NaN: their entries of C are
// computed in IEEE FP64 after the emulated product (which leaves them alone).
template <typename T>
cudaError_t launch_nonfinite_patch(const GemmArgs<T>& g, const ViewT<T>& va, const ViewT<T>& vb, const Layout& L,
                                   uint8_t* w, cudaStream_t st) {
    const int* cnta = reinterpret_cast<const int*>(w + L.cnta_off);
    const int* cntb = reinterpret_cast<const int*>(w + L.cntb_off);
    cudaError_t e = launch_dependent(ozaki_nonfinite_patch<T>, dim3(2 * sm_count_cached()), dim3(256), 0, st, va, vb,
                                     g.m, g.n, g.k, (double)g.alpha, (double)g.beta, g.c, g.ldc, cnta,
                                     reinterpret_cast<const int*>(w + L.lista_off), cntb,
                                     reinterpret_cast<const int*>(w + L.listb_off),
                                     reinterpret_cast<const int*>(w + L.expa_off),
                                     reinterpret_cast<const int*>(w + L.status_off));
    count_launch();
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename T>
cudaError_t gemm_ozaki_crt(const GemmArgs<T>& g, const OzakiPlan& p, void* ws, cudaStream_t st, bool a_ready) {
    const Layout L = ozaki_layout(p);
    uint8_t* w = static_cast<uint8_t*>(ws);
    int8_t* a_planes = reinterpret_cast<int8_t*>(w + L.a_planes_off);
    int8_t* b_planes = reinterpret_cast<int8_t*>(w + L.b_planes_off);
    int8_t* residues = reinterpret_cast<int8_t*>(w + L.res_off);
    auto* maxa = reinterpret_cast<unsigned long long*>(w + L.maxa_off);
    auto* maxb = reinterpret_cast<unsigned long long*>(w + L.maxb_off);
    auto* suma = reinterpret_cast<double*>(w + L.suma_off);
    auto* sumb = reinterpret_cast<double*>(w + L.sumb_off);
    int* expa = reinterpret_cast<int*>(w + L.expa_off);
    int* expb = reinterpret_cast<int*>(w + L.expb_off);
    int* cnta = reinterpret_cast<int*>(w + L.cnta_off);
    int* cntb = reinterpret_cast<int*>(w + L.cntb_off);
    int* lista = reinterpret_cast<int*>(w + L.lista_off);
    int* listb = reinterpret_cast<int*>(w + L.listb_off);
    int* status = reinterpret_cast<int*>(w + L.status_off);
    const int nmod = p.moduli;
    const CrtHost& H = crt_host(nmod);
    g_last_moduli.store(nmod);

    ViewT<T> va{g.a, g.transa == 'N' ? 1 : g.lda, g.transa == 'N' ? g.lda : 1, g.m, g.k};
    ViewT<T> vb{g.b, g.transb == 'N' ? g.ldb : 1, g.transb == 'N' ? 1 : g.ldb, g.n, g.k};
    // op(B)^T is op(A) itself (C = A A^T or A^T A, as SYRK asks): op(B)'s planes,
    // exponents and Inf / NaN list are op(A)'s, so they are computed once
    const bool same = !a_ready && p.pair && p.m_pad == p.n_pad && g.m == g.n && g.a == g.b && g.lda == g.ldb &&
                      ((g.transa == 'N') != (g.transb == 'N'));
    const int sides = same ? 1 : 2;
    // triangle mode (CTA-pair kernel): only the tiles meeting the stored triangle of C
    const int tri = p.pair ? g.tri : 0;
    // a_ready: op(A)'s statistics, exponents, Inf / NaN row list and planes stay;
    // op(B)'s accumulators, its list count and the status word are cleared
    cudaError_t e = a_ready ? cudaMemsetAsync(w + L.maxb_off, 0, L.b_clear_end - L.maxb_off, st)
                            : cudaMemsetAsync(w, 0, L.b_clear_end, st);
    if (e != cudaSuccess) return e;
    for (int side = a_ready ? 1 : 0; side < sides; ++side) {
        const ViewT<T>& v = side ? vb : va;
        const dim3 grid = v.rs == 1 ? dim3((v.rows + 255) / 256, (v.cols + 63) / 64)
                                    : dim3((v.rows + 7) / 8, (v.cols + 1023) / 1024);
        // the first pass follows the memset of the statistics: an ordinary launch
        if (side == (a_ready ? 1 : 0))
            ozaki_absmax<T><<<grid, 256, 0, st>>>(v, side ? maxb : maxa, side ? sumb : suma);
        else if ((e = launch_dependent(ozaki_absmax<T>, grid, dim3(256), 0, st, v, side ? maxb : maxa,
                                       side ? sumb : suma)) != cudaSuccess)
            return e;
        count_launch();
    }
    for (int side = a_ready ? 1 : 0; side < sides; ++side) {
        const ViewT<T>& v = side ? vb : va;
        const int rows_pad = side ? p.n_pad : p.m_pad;
        dim3 sgrid(p.k_pad / 128, rows_pad / 32);
        if ((e = launch_dependent(ozaki_crt_split<T>, sgrid, dim3(256), 0, st, v, (const unsigned long long*)(side ? maxb : maxa),
                                  (const double*)(side ? sumb : suma), H.P, nmod, rows_pad, p.k_pad,
                                  side ? b_planes : a_planes, side ? expb : expa, side ? cntb : cnta,
                                  side ? listb : lista)) != cudaSuccess)
            return e;
        count_launch();
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (same) {  // op(B)'s column exponents and Inf / NaN list are op(A)'s row ones
        if ((e = cudaMemcpyAsync(expb, expa, (size_t)p.n_pad * sizeof(int), cudaMemcpyDeviceToDevice, st)) !=
                cudaSuccess ||
            (e = cudaMemcpyAsync(cntb, cnta, sizeof(int), cudaMemcpyDeviceToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(listb, lista, (size_t)g.n * sizeof(int), cudaMemcpyDeviceToDevice, st)) !=
                cudaSuccess)
            return e;
    }

    CUtensorMap ma, mb;
    if ((e = make_map(&ma, a_planes, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, p.k_pad, (long)nmod * p.m_pad, kUM)) !=
        cudaSuccess)
        return e;
    if ((e = make_map(&mb, same ? a_planes : b_planes, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, p.k_pad,
                      (long)nmod * p.n_pad, p.pair ? kUN / 2 : kUN)) != cudaSuccess)
        return e;

    UmmaParams P{};
    P.m = g.m;
    P.n = g.n;
    P.m_pad = p.m_pad;
    P.n_pad = p.n_pad;
    P.k_chunks = p.k_pad / kChunkBytes;
    P.kseg_chunks = P.k_chunks;  // k <= kCrtMaxK: one INT32 segment
    P.num_kseg = 1;
    P.tiles_m = p.m_pad / (p.pair ? 2 * kUM : kUM);
    P.tiles_n = p.n_pad / kUN;
    P.num_tiles = P.tiles_m * P.tiles_n;
    // one modulus per job; jobs alternate between the two TMEM accumulators so
    // the epilogue of modulus l overlaps the products of modulus l + 1
    P.num_jobs = nmod;
    for (int l = 0; l < nmod; ++l) {
        P.job_first_step[l] = l;
        P.job_num_steps[l] = 1;
        P.job_groups[l] = 1;
        P.job_shift[l][0] = l;
        P.job_shift[l][1] = 0;
        P.job_buf[l] = l & 1;
        P.step_a[l] = l;
        P.step_b[l] = l;
        P.step_acc[l] = l & 1;
    }
    P.status = status;
    P.residues = residues;
    P.res_plane = (long)p.m_pad * p.n_pad;
    // CTA pair, modulus-major: bands of tile-rows whose A rows of one modulus
    // (band x 256 rows x k_pad bytes) stay within ~48 MB of L2 while the band
    // sweeps the tile-columns
    static const long band_bytes = [] {
        const char* v = std::getenv("ZYNUM_GPU_CRT_BAND_MB");
        const long mb = v ? std::atol(v) : 48;
        return (mb >= 4 && mb <= 120 ? mb : 48) << 20;
    }();
    P.band_rows = (int)std::max(1L, std::min<long>(P.tiles_m, band_bytes / (256L * p.k_pad)));
    if (tri && P.tiles_m == P.tiles_n) {  // the tiles meeting the stored triangle only
        P.tri = tri;
        P.num_tiles = P.tiles_m * (P.tiles_m + 1) / 2;
    }
    if ((e = set_wait_params(P, p.hold)) != cudaSuccess) return e;
    // after op(A)'s exponents and lists were copied to op(B)'s (one operand split once) the
    // kernel before the products is a copy: an ordinary launch
    e = p.pair ? launch_umma_2cta<KIND_I8, EPI_RESIDUE>(ma, mb, P, st, !same)
               : launch_umma<KIND_I8, EPI_RESIDUE>(ma, mb, P, st, !same);
    if (e != cudaSuccess) return e;

    dim3 cgrid((g.m + 15) / 16, (g.n + 127) / 128);
    if ((e = launch_dependent(combine_at<kCrtMaxModuli, T>(nmod), cgrid, dim3(256), 0, st, (const int8_t*)residues,
                              P.res_plane, p.n_pad, g.m, g.n, (const int*)expa, (const int*)expb, (double)g.alpha,
                              (double)g.beta, g.c, (long)g.ldc, H.K, (const int*)status, tri)) != cudaSuccess)
        return e;
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_nonfinite_patch(g, va, vb, L, w, st);
}
}  // namespace

int ozaki_crt_bits(int moduli) {
    if (moduli < 1 || moduli > kCrtMaxModuli) return 0;
    return crt_host(moduli).P;
}
int ozaki_last_moduli() { return g_last_moduli.load(); }

int sgemm_crt_moduli(int k) {
    // scaling bits P >= 25 + log2(sqrt(k)): a row whose entries all have the
    // magnitude of its largest has 2-norm max sqrt(k), so every such entry keeps
    // its 24-bit significand and a guard bit
    const double need = 25.0 + 0.5 * std::log2((double)std::max(k, 1));
    for (int n = 2; n <= kCrtMaxModuli; ++n)
        if (crt_host(n).P >= need) return n;
    return kCrtMaxModuli;
}

cudaError_t sgemm_ozaki(const GemmArgsF32& g, const OzakiPlan& p, void* ws, cudaStream_t st) {
    if (p.scheme != OZAKI_CRT || g.k > kCrtMaxK) return cudaErrorInvalidValue;
    return gemm_ozaki_crt<float>(g, p, ws, st, false);
}

cudaError_t dgemm_ozaki(const GemmArgsF64& g, const OzakiPlan& plan, void* ws, cudaStream_t st, bool a_ready) {
    if (plan.scheme == OZAKI_CRT) return gemm_ozaki_crt<double>(g, plan, ws, st, a_ready);
    // the slice scheme (its slice count depends on both operands) always recomputes op(A)
    OzakiPlan p = plan;
    const Layout L = ozaki_layout(p);
    uint8_t* w = static_cast<uint8_t*>(ws);
    int8_t* a_planes = reinterpret_cast<int8_t*>(w + L.a_planes_off);
    int8_t* b_planes = reinterpret_cast<int8_t*>(w + L.b_planes_off);
    auto* maxa = reinterpret_cast<unsigned long long*>(w + L.maxa_off);
    auto* maxb = reinterpret_cast<unsigned long long*>(w + L.maxb_off);
    auto* suma = reinterpret_cast<double*>(w + L.suma_off);
    auto* sumb = reinterpret_cast<double*>(w + L.sumb_off);
    int* expa = reinterpret_cast<int*>(w + L.expa_off);
    int* expb = reinterpret_cast<int*>(w + L.expb_off);
    float* spread = reinterpret_cast<float*>(w + L.spread_off);
    int* status = reinterpret_cast<int*>(w + L.status_off);
    int* cnta = reinterpret_cast<int*>(w + L.cnta_off);
    int* cntb = reinterpret_cast<int*>(w + L.cntb_off);
    int* lista = reinterpret_cast<int*>(w + L.lista_off);
    int* listb = reinterpret_cast<int*>(w + L.listb_off);

    // op(A) as rows i / cols p; op(B)^T as rows j / cols p.
    View va{g.a, g.transa == 'N' ? 1 : g.lda, g.transa == 'N' ? g.lda : 1, g.m, g.k};
    View vb{g.b, g.transb == 'N' ? g.ldb : 1, g.transb == 'N' ? 1 : g.ldb, g.n, g.k};

    cudaError_t e = cudaMemsetAsync(w, 0, L.b_clear_end, st);  // the slice scheme recomputes both operands
    if (e != cudaSuccess) return e;
    for (int side = 0; side < 2; ++side) {
        const View& v = side ? vb : va;
        if (v.rs == 1) {
            dim3 grid((v.rows + 255) / 256, (v.cols + 63) / 64);
            ozaki_absmax<<<grid, 256, 0, st>>>(v, side ? maxb : maxa, side ? sumb : suma);
        } else {
            dim3 grid((v.rows + 7) / 8, (v.cols + 1023) / 1024);
            ozaki_absmax<<<grid, 256, 0, st>>>(v, side ? maxb : maxa, side ? sumb : suma);
        }
        count_launch();
    }
    if (p.slices <= 0) {
        // Automatic slice count from the data's dynamic range (one small
        // device -> host read; the stream is synchronised here).
        ozaki_spread<<<1, 1024, 0, st>>>(maxa, suma, g.m, g.k, spread);
        count_launch();
        ozaki_spread<<<1, 1024, 0, st>>>(maxb, sumb, g.n, g.k, spread + 1);
        count_launch();
        float h[2] = {0.f, 0.f};
        if ((e = cudaMemcpyAsync(h, spread, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
        p.slices = ozaki_auto_slices(h[0], h[1]);
    }
    g_last_slices.store(p.slices);
    for (int side = 0; side < 2; ++side) {
        const View& v = side ? vb : va;
        const int rows_pad = side ? p.n_pad : p.m_pad;
        dim3 sgrid(p.k_pad / 128, rows_pad / 32);
        ozaki_split<<<sgrid, 256, 0, st>>>(v, side ? maxb : maxa, p.slices, rows_pad, p.k_pad,
                                           side ? b_planes : a_planes, side ? expb : expa, side ? cntb : cnta,
                                           side ? listb : lista);
        count_launch();
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;

    CUtensorMap ma, mb;
    if ((e = make_map(&ma, a_planes, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, p.k_pad, (long)p.slices * p.m_pad, kUM)) !=
        cudaSuccess)
        return e;
    if ((e = make_map(&mb, b_planes, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, p.k_pad, (long)p.slices * p.n_pad,
                      p.pair ? kUN / 2 : kUN)) != cudaSuccess)
        return e;

    UmmaParams P{};
    P.m = g.m;
    P.n = g.n;
    P.m_pad = p.m_pad;
    P.n_pad = p.n_pad;
    P.k_chunks = p.k_pad / kChunkBytes;
    P.kseg_chunks = max_kseg_chunks(p.slices);
    if (P.kseg_chunks > P.k_chunks) P.kseg_chunks = P.k_chunks;
    P.num_kseg = (P.k_chunks + P.kseg_chunks - 1) / P.kseg_chunks;
    P.tiles_m = p.m_pad / (p.pair ? 2 * kUM : kUM);
    P.tiles_n = p.n_pad / kUN;
    P.num_tiles = P.tiles_m * P.tiles_n;
    // Groups g = s+1 .. 2 (smallest contributions first), two per job: the
    // job's steps walk t upwards emitting (t, g_a - t) then (t, g_b - t), so
    // consecutive steps share A_t or B_{g_b - t}.
    int nsteps = 0, njobs = 0;
    for (int ga = p.slices + 1; ga >= 2; ga -= 2) {
        const int gb = ga - 1;
        const bool two = gb >= 2;
        P.job_first_step[njobs] = nsteps;
        P.job_groups[njobs] = two ? 2 : 1;
        P.job_shift[njobs][0] = 7 * ga;
        P.job_shift[njobs][1] = two ? 7 * gb : 0;
        for (int t = 1; t <= p.slices; ++t) {
            for (int h = 0; h < (two ? 2 : 1); ++h) {
                const int u = (h ? gb : ga) - t;
                if (u < 1 || u > p.slices) continue;
                P.step_a[nsteps] = t - 1;
                P.step_b[nsteps] = u - 1;
                P.step_acc[nsteps] = h;
                ++nsteps;
            }
        }
        P.job_num_steps[njobs] = nsteps - P.job_first_step[njobs];
        ++njobs;
    }
    P.num_jobs = njobs;
    P.alpha = g.alpha;
    P.beta = g.beta;
    P.c = g.c;
    P.ldc = g.ldc;
    P.row_exp = expa;
    P.col_exp = expb;
    P.status = status;
    if ((e = set_wait_params(P, p.hold)) != cudaSuccess) return e;
    e = p.pair ? launch_umma_2cta<KIND_I8, EPI_OZAKI_F64>(ma, mb, P, st)
               : launch_umma<KIND_I8, EPI_OZAKI_F64>(ma, mb, P, st);
    if (e != cudaSuccess) return e;
    return launch_nonfinite_patch(g, va, vb, L, w, st);
}

cudaError_t wait_report_word(int** out) {
    cudaError_t e = report_word(out);
    if (e == cudaSuccess) g_products_launched.store(true);
    return e;
}

int ozaki_take_wait_report(cudaStream_t stream, cudaError_t* err) {
    *err = cudaSuccess;
    if (!g_products_launched.load()) return 0;
    int* word = nullptr;
    cudaError_t e = report_word(&word);
    int v = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&v, word, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && v != 0) e = cudaMemsetAsync(word, 0, sizeof(int), stream);
    if (e == cudaSuccess && v != 0) e = cudaStreamSynchronize(stream);
    *err = e;
    return e == cudaSuccess ? v : 0;
}

size_t bf16x3_workspace_bytes(int m, int n, int k) {
    const long mp = round_up(m, use_cta_pair(m) ? 2 * kUM : kUM), np = round_up(n, kUN), kp = round_up(k, 128);
    return (size_t)(2 * mp * kp * 2 + 2 * np * kp * 2 + 1024);
}

cudaError_t sgemm_bf16x3(const GemmArgsF32& g, void* ws, cudaStream_t st) {
    // K is padded to 128 elements: the split kernel writes 128 columns per block.
    const bool pair = use_cta_pair(g.m);
    const int mp = (int)round_up(g.m, pair ? 2 * kUM : kUM), np = (int)round_up(g.n, kUN), kp = (int)round_up(g.k, 128);
    __nv_bfloat16* a_planes = static_cast<__nv_bfloat16*>(ws);
    __nv_bfloat16* b_planes = a_planes + 2L * mp * kp;
    ViewF va{g.a, g.transa == 'N' ? 1 : g.lda, g.transa == 'N' ? g.lda : 1, g.m, g.k};
    ViewF vb{g.b, g.transb == 'N' ? g.ldb : 1, g.transb == 'N' ? 1 : g.ldb, g.n, g.k};
    bf16_split<<<dim3((kp + 127) / 128, mp / 32), 256, 0, st>>>(va, mp, kp, a_planes);
    count_launch();
    bf16_split<<<dim3((kp + 127) / 128, np / 32), 256, 0, st>>>(vb, np, kp, b_planes);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    CUtensorMap ma, mb;
    if ((e = make_map(&ma, a_planes, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, kp, 2L * mp, kUM)) != cudaSuccess) return e;
    if ((e = make_map(&mb, b_planes, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, kp, 2L * np, pair ? kUN / 2 : kUN)) !=
        cudaSuccess)
        return e;
    UmmaParams P{};
    P.m = g.m;
    P.n = g.n;
    P.m_pad = mp;
    P.n_pad = np;
    P.k_chunks = kp / 64;
    P.kseg_chunks = P.k_chunks;
    P.num_kseg = 1;
    P.tiles_m = mp / (pair ? 2 * kUM : kUM);
    P.tiles_n = np / kUN;
    P.num_tiles = P.tiles_m * P.tiles_n;
    // one job, one FP32 accumulator: hi*lo, hi*hi, lo*hi (consecutive steps
    // share an operand); plane 0 = hi, 1 = lo
    P.num_jobs = 1;
    P.job_first_step[0] = 0;
    P.job_num_steps[0] = 3;
    P.job_groups[0] = 1;
    P.job_shift[0][0] = 0;
    P.job_shift[0][1] = 0;
    const int sa[3] = {0, 0, 1}, sb[3] = {1, 0, 0};
    for (int q = 0; q < 3; ++q) {
        P.step_a[q] = sa[q];
        P.step_b[q] = sb[q];
        P.step_acc[q] = 0;
    }
    P.alpha_f = g.alpha;
    P.beta_f = g.beta;
    P.c = g.c;
    P.ldc = g.ldc;
    if ((e = set_wait_params(P, false)) != cudaSuccess) return e;
    if (pair) return launch_umma_2cta<KIND_BF16, EPI_F32>(ma, mb, P, st);
    return launch_umma<KIND_BF16, EPI_F32>(ma, mb, P, st);
}

}  // namespace zb
