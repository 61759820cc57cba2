// passtc.cuh -- strided x / y passes whose line transforms run on the tensor
// cores as split-TF32 DFT-matrix GEMMs (FP32, N = 256 and 512).
//
// Same contract as k_passr / k_pass (PassSpec / PassPtrs: tiles of columns x N
// rows, kept / compact rows and outer indices, up to two outputs per tile,
// each the transform of the tile times a spectral multiplier, optional dealias
// mask), for tiles of NB = 8 columns.  A length-N transform, N = N1 N2 with
// N2 = 16, n = N2 n1 + n2, k = k1 + N1 k2, is
//   step 1  Y[n2][k1] = sum_n1 x[N2 n1 + n2] W_N1^(n1 k1)         (DFT-N1 GEMM)
//   twiddle Y[n2][k1] *= W_N^(n2 k1)
//   step 3  X[k1 + N1 k2] = sum_n2 Y[n2][k1] W_N2^(n2 k2)         (DFT-N2 GEMM)
// Each step is a real GEMM D = A B on tcgen05 (kind::tf32, M = 128, F32
// accumulators in TMEM): the rows of A are the (column, n2) or (column, k1)
// lines of the tile, its K index the real and imaginary parts of the line,
// and B the real form [[Re W, Im W], [-Im W, Re W]] of the DFT matrix.  FP32
// accuracy comes from three products per GEMM: with a = a_hi + a_lo (a_hi the
// value rounded to TF32, a_lo the exact remainder, read as TF32 by the MMA)
// and likewise b, D = a_hi b_hi + a_lo b_hi + a_hi b_lo, which leaves out only
// a_lo b_lo (relative 2^-22).
//
// Per tile (and per output of a tile), 16 warps:
//   P1  load the rows of the tile from global memory (issued one tile ahead,
//       into registers), apply the mask and the multiplier, split, and write
//       A1 (16-byte stores of 4 consecutive n1);
//   MMA step 1 (3 x 2N1/8 MMAs of 128 x 2N1 x 8), committed to mbarrier 0;
//   P2  output of the previous tile while step 1 runs: D3 rows from TMEM into
//       an output tile (in A3's shared memory) and coalesced row stores;
//   P3  D1 rows from TMEM, twiddle, split, write A3;
//   MMA step 3 (per 128-row M tile, 3 x 4 MMAs of 128 x 32 x 8), committed to
//       mbarrier 1 -- it runs while P1 of the next tile builds A1.
// Waits on the mbarriers are bounded: one that runs out sets bit 1 of *err
// (err may be null: no report), waits (bounded) for the MMAs in flight, frees
// the TMEM and leaves.
//
// Index maps (NB = 8 columns c of the tile):
//   A1 row m1 = c + 8 n2 (128 rows), K index n1 (Re) or N1 + n1 (Im);
//   D1 row m1 = TMEM lane, column k1 (Re) or N1 + k1 (Im);
//   A3 M tile k1 / 16, row c + 8 (k1 % 16), K index n2 (Re) or N2 + n2 (Im);
//   D3 row = that, column k2 (Re) or N2 + k2 (Im), at TMEM column 2 N1 + 32 * tile.
// Operands are K-major without swizzle: core matrices of 8 rows x 4 K values
// (128 bytes, a row's 16 bytes contiguous), the K chunks of a core-matrix row
// group 128 bytes apart (leading byte offset), row groups K * 4 * 4 bytes apart
// (stride byte offset); an MMA (K = 8) reads two chunks.  Row r % 8 of a core
// matrix is 16 bytes at (r % 8) * 16, so the 8 lanes that own the 8 columns of
// the tile (A1, 16-byte stores) or, with the column and n2 % 4, the 32 words
// of a row group's chunk (A3, 4-byte stores) hit distinct banks.
#pragma once
#include "passreg.cuh"
#include "tcgen05.cuh"

#include <type_traits>

namespace gnss {

__host__ __device__ constexpr bool ptc_size(int n) { return n == 256 || n == 512; }

template <int N> struct PTCfg {
    static_assert(ptc_size(N), "tensor-core passes serve N = 256, 512");
    static constexpr int NB = 8;                 // columns per tile
    static constexpr int N2 = 16;
    static constexpr int N1 = N / N2;            // 32 or 16
    static constexpr int NT = 512;               // 16 warps
    static constexpr int K1 = 2 * N1;            // step-1 K and N (Re and Im)
    static constexpr int K3 = 2 * N2;            // step-3 K and N
    static constexpr int MT3 = N1 * NB / 128;    // step-3 M tiles (2 or 1)
    static constexpr int KG1 = K1 / 8, KG3 = K3 / 8;   // K groups: one MMA (K = 8) each
    static constexpr int A1_BYTES = 128 * K1 * 4;      // one of hi / lo
    static constexpr int A3_TILE = 128 * K3 * 4;
    static constexpr int A3_BYTES = MT3 * A3_TILE;
    static constexpr int B1_BYTES = K1 * K1 * 4, B3_BYTES = K3 * K3 * 4;
    static constexpr int B1_SBO = (K1 / 4) * 128, B3_SBO = (K3 / 4) * 128;
    static constexpr int A1_SBO = B1_SBO, A3_SBO = B3_SBO;   // row-group strides of the A operands
    static constexpr int OFF_A1H = 0, OFF_A1L = A1_BYTES;
    static constexpr int OFF_A3H = 2 * A1_BYTES, OFF_A3L = OFF_A3H + A3_BYTES;
    static constexpr int OFF_B1H = OFF_A3L + A3_BYTES, OFF_B1L = OFF_B1H + B1_BYTES;
    static constexpr int OFF_B3H = OFF_B1L + B1_BYTES, OFF_B3L = OFF_B3H + B3_BYTES;
    static constexpr int OFF_TW = OFF_B3L + B3_BYTES;  // N twiddles W_N^j (signed)
    static constexpr int OFF_MISC = OFF_TW + N * 8;    // 2 mbarriers, TMEM address, dmax[NB]
    static constexpr int OFF_OROW = OFF_MISC + 64;     // N destination row offsets
    static constexpr int SMEM = OFF_OROW + N * 4 + 1024;   // + slack to align the base to 1024 bytes
    static constexpr int LDO = NB;                     // output tile row pitch (complex), in A3's space
    static constexpr uint32_t D1_COL = 0, D3_COL = K1;
    static constexpr uint32_t TCOLS = (K1 + MT3 * K3) <= 64 ? 64u : 128u;
    static constexpr int NIT = N1 / 16;                // P1: groups of 4 rows per thread
    static constexpr int KQ = N1 / 4;                  // P3: k1 per thread
    static_assert(N * LDO * 8 <= A3_BYTES, "output tile fits in A3");
    static_assert(K1 + MT3 * K3 <= (int)TCOLS, "TMEM columns");
};

template <int N, int SIGN, bool MB = false>
__global__ void __launch_bounds__(512, 1)
k_passtc(const __grid_constant__ PassPtrs<float> P, const __grid_constant__ PassSpec sp,
         const float2 *__restrict__ tw, unsigned *__restrict__ err) {
    using C = PTCfg<N>;
    using V = float2;
    constexpr int NB = C::NB, N1 = C::N1, N2 = C::N2, NIT = C::NIT, KQ = C::KQ;
    pdl_wait();   // before the prologue too: its TMEM allocation waits for the previous kernel's blocks
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t raw_addr = smem_u32(smem_raw);
    const uint32_t base = (raw_addr + 1023u) & ~1023u;
    unsigned char *sm = smem_raw + (base - raw_addr);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = sp.outer.count() * sp.ncolblk;
    const int mitems = sp.nin * ntiles;      // items of one member
    const int nitems = MB ? sp.nmem * mitems : mitems;   // < 2^31 (members x inputs x outer indices x column blocks)
    int item = blockIdx.x;
    if (item >= nitems) return;   // uniform for the block
    V *twl = reinterpret_cast<V *>(sm + C::OFF_TW);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + C::OFF_MISC);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + C::OFF_MISC + 16);
    int *dmax_s = reinterpret_cast<int *>(sm + C::OFF_MISC + 32);
    int *orow = reinterpret_cast<int *>(sm + C::OFF_OROW);
    V *outt = reinterpret_cast<V *>(sm + C::OFF_A3H);   // output tile (A3's space between the steps)

    // ---- set-up: signed twiddles, the DFT matrices (split), destination rows, barriers, TMEM
    for (int i = tid; i < N; i += C::NT) {
        const V t = tw[i];
        twl[i] = SIGN < 0 ? t : V{t.x, -t.y};
        int o = -1;   // destination offset of output row i (elements; < 2^31 per tile)
        if (sp.row_out.kept(i)) o = (sp.row_out_compact ? sp.row_out.compact(i) : i) * (int)sp.d_row;
        orow[i] = o;
    }
    __syncthreads();
    auto put_b = [&](int off_h, int off_l, int sbo, int kk, int n, float val) {
        const int o = (n & 7) * 16 + (n >> 3) * sbo + (kk & 3) * 4 + (kk >> 2) * 128;
        float hi, lo;
        tc::split_tf32(val, hi, lo);
        *reinterpret_cast<float *>(sm + off_h + o) = hi;
        *reinterpret_cast<float *>(sm + off_l + o) = lo;
    };
    // B[kk][n]: kk = Re / Im of the input index, n = Re / Im of the output index
    for (int i = tid; i < C::K1 * C::K1; i += C::NT) {
        const int kk = i / C::K1, n = i - kk * C::K1;
        const int a = kk % N1, b = n % N1;
        const V w = twl[(N2 * a * b) % N];   // W_N1^(a b)
        const float v = (kk < N1) == (n < N1) ? w.x : (kk < N1 ? w.y : -w.y);
        put_b(C::OFF_B1H, C::OFF_B1L, C::B1_SBO, kk, n, v);
    }
    for (int i = tid; i < C::K3 * C::K3; i += C::NT) {
        const int kk = i / C::K3, n = i - kk * C::K3;
        const int a = kk % N2, b = n % N2;
        const V w = twl[(N1 * a * b) % N];   // W_N2^(a b)
        const float v = (kk < N2) == (n < N2) ? w.x : (kk < N2 ? w.y : -w.y);
        put_b(C::OFF_B3H, C::OFF_B3L, C::B3_SBO, kk, n, v);
    }
    if (warp == 0) tc::alloc(tslot, C::TCOLS);
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    fence_proxy_async_smem();   // B matrices written by threads, read by the MMAs
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const WaitCtl wc(err);

    auto decode = [&](int it, int &mi, int &fi, int &oc, int &o, int &c0) {
        mi = MB ? it / mitems : 0;   // member of a batch (MB)
        const int r = MB ? it - mi * mitems : it;
        fi = r / ntiles;
        const int t = r - fi * ntiles;
        oc = t / sp.ncolblk;
        o = sp.outer.expand(oc);
        c0 = (t - oc * sp.ncolblk) * NB;
    };

    // ---- P1 geometry: column pc, rows N2 (4 a + e) + pn2 (e < 4) for a = pa0 + 4 it, it < NIT.
    // The source offsets of these rows (r s_row, or -1 where the spec keeps no row) are fixed for the launch.
    const int pc = lane & 7, pn2 = (lane >> 3) + 4 * (warp & 3), pa0 = warp >> 2;
    int roff[NIT][4];
#pragma unroll
    for (int it = 0; it < NIT; ++it)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int row = N2 * (4 * (pa0 + 4 * it) + e) + pn2;
            roff[it][e] = sp.row_in.kept(row) ? (sp.row_in_compact ? sp.row_in.compact(row) : row) * (int)sp.s_row
                                              : -1;
        }
    V raw[NIT][4];
    auto load = [&](int it_item) {
        int mi, fi, oc, o, c0;
        decode(it_item, mi, fi, oc, o, c0);
        const V *src = P.in[fi] + (MB ? mi * sp.ms_in : 0LL) + (long long)(sp.outer_in_compact ? oc : o) * sp.s_out + c0 + pc;
        const bool col_ok = c0 + pc < sp.ncols;
#pragma unroll
        for (int it = 0; it < NIT; ++it)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                raw[it][e] = (col_ok && roff[it][e] >= 0) ? __ldg(src + roff[it][e]) : V{0.f, 0.f};
    };
    // A1 from the loaded rows: mask, multiplier (fixed per output), split, 16-byte stores of 4 consecutive n1
    // of row m1 = pc + 8 pn2
    auto build_a1_mul = [&](auto mulc, int c0, double k_out) {
        constexpr int MUL = decltype(mulc)::value;
        const int dmax = sp.mask ? dmax_s[pc] : N;
        const double kcd = wavenum(c0 + pc, sp.n_col, sp.dk_col);
        const float kk = MUL == V_IK_OUT ? (float)k_out : (float)kcd;
        const float dkr = (float)sp.dk_row;
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const int a = pa0 + 4 * it;
            float rh[4], rl[4], ih[4], il[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int row = N2 * (4 * a + e) + pn2;
                V x = raw[it][e];
                if (row_dist<N>(row) > dmax) x = V{0.f, 0.f};
                if constexpr (MUL == V_IK_ROW) {
                    const float kr = dkr * (float)(row < N / 2 ? row : row - N);
                    x = V{-kr * x.y, kr * x.x};
                } else if constexpr (MUL == V_IK_OUT || MUL == V_IK_COL) {
                    x = V{-kk * x.y, kk * x.x};
                } else if constexpr (MUL == V_LAP) {
                    const float k2 = (float)ksq3(wavenum(row, N, sp.dk_row), k_out, kcd);
                    x = V{-k2 * x.x, -k2 * x.y};
                }
                tc::split_tf32(x.x, rh[e], rl[e]);
                tc::split_tf32(x.y, ih[e], il[e]);
            }
            const int o_re = pc * 16 + pn2 * C::A1_SBO + a * 128;
            const int o_im = o_re + (N1 / 4) * 128;
            *reinterpret_cast<float4 *>(sm + C::OFF_A1H + o_re) = make_float4(rh[0], rh[1], rh[2], rh[3]);
            *reinterpret_cast<float4 *>(sm + C::OFF_A1L + o_re) = make_float4(rl[0], rl[1], rl[2], rl[3]);
            *reinterpret_cast<float4 *>(sm + C::OFF_A1H + o_im) = make_float4(ih[0], ih[1], ih[2], ih[3]);
            *reinterpret_cast<float4 *>(sm + C::OFF_A1L + o_im) = make_float4(il[0], il[1], il[2], il[3]);
        }
    };
    auto build_a1 = [&](int mul, int c0, double k_out) {
        switch (mul) {
            case V_IK_ROW: build_a1_mul(std::integral_constant<int, V_IK_ROW>{}, c0, k_out); break;
            case V_IK_OUT: build_a1_mul(std::integral_constant<int, V_IK_OUT>{}, c0, k_out); break;
            case V_IK_COL: build_a1_mul(std::integral_constant<int, V_IK_COL>{}, c0, k_out); break;
            case V_LAP: build_a1_mul(std::integral_constant<int, V_LAP>{}, c0, k_out); break;
            default: build_a1_mul(std::integral_constant<int, V_ONE>{}, c0, k_out); break;
        }
    };
    auto issue_step1 = [&]() {
        tc::fence_after_sync();
        constexpr uint32_t id = tc::idesc_tf32(128, C::K1, 0);
#pragma unroll 1
        for (int kg = 0; kg < C::KG1; ++kg) {
            const uint64_t ah = tc::smem_desc(base + C::OFF_A1H + kg * 256, 128, C::A1_SBO, tc::LAYOUT_NONE);
            const uint64_t al = tc::smem_desc(base + C::OFF_A1L + kg * 256, 128, C::A1_SBO, tc::LAYOUT_NONE);
            const uint64_t bh = tc::smem_desc(base + C::OFF_B1H + kg * 256, 128, C::B1_SBO, tc::LAYOUT_NONE);
            const uint64_t bl = tc::smem_desc(base + C::OFF_B1L + kg * 256, 128, C::B1_SBO, tc::LAYOUT_NONE);
            tc::mma_tf32(tmem + C::D1_COL, ah, bh, id, kg > 0 ? 1u : 0u);
            tc::mma_tf32(tmem + C::D1_COL, al, bh, id, 1u);
            tc::mma_tf32(tmem + C::D1_COL, ah, bl, id, 1u);
        }
        tc::commit(&bar[0]);
    };
    auto issue_step3 = [&]() {
        tc::fence_after_sync();
        constexpr uint32_t id = tc::idesc_tf32(128, C::K3, 0);
#pragma unroll 1
        for (int t = 0; t < C::MT3; ++t) {
#pragma unroll 1
            for (int kg = 0; kg < C::KG3; ++kg) {
                const int ao = t * C::A3_TILE + kg * 256;
                const uint64_t ah = tc::smem_desc(base + C::OFF_A3H + ao, 128, C::A3_SBO, tc::LAYOUT_NONE);
                const uint64_t al = tc::smem_desc(base + C::OFF_A3L + ao, 128, C::A3_SBO, tc::LAYOUT_NONE);
                const uint64_t bh = tc::smem_desc(base + C::OFF_B3H + kg * 256, 128, C::B3_SBO, tc::LAYOUT_NONE);
                const uint64_t bl = tc::smem_desc(base + C::OFF_B3L + kg * 256, 128, C::B3_SBO, tc::LAYOUT_NONE);
                const uint32_t d = tmem + C::D3_COL + t * C::K3;
                tc::mma_tf32(d, ah, bh, id, kg > 0 ? 1u : 0u);
                tc::mma_tf32(d, al, bh, id, 1u);
                tc::mma_tf32(d, ah, bl, id, 1u);
            }
        }
        tc::commit(&bar[1]);
    };
    // P3: D1 -> twiddle -> split -> A3.  Thread: TMEM lane m1 = 32 q + lane (c = lane % 8,
    // n2 = 4 q + lane / 8), k1 in [part KQ, part KQ + KQ); 4-byte stores into rows c + 8 (k1 % 16)
    auto build_a3 = [&]() {
        const int q = warp & 3, part = warp >> 2;
        const int c = lane & 7, n2 = 4 * q + (lane >> 3);
        float yr[KQ], yi[KQ];
        const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + C::D1_COL + part * KQ;
        if constexpr (KQ == 8) {
            tc::ld_x8(ta, yr);
            tc::ld_x8(ta + N1, yi);
        } else {
            tc::ld_x4(ta, yr);
            tc::ld_x4(ta + N1, yi);
        }
        tc::wait_ld();
        const int o_re = c * 16 + (n2 >> 2) * 128 + (n2 & 3) * 4;
        const int o_im = o_re + (N2 / 4) * 128;
#pragma unroll
        for (int i = 0; i < KQ; ++i) {
            const int k1 = part * KQ + i;
            const V w = twl[(n2 * k1) & (N - 1)];
            const float a = yr[i] * w.x - yi[i] * w.y, b = yr[i] * w.y + yi[i] * w.x;
            float rh, rl, ih, il;
            tc::split_tf32(a, rh, rl);
            tc::split_tf32(b, ih, il);
            const int rb = (k1 >> 4) * C::A3_TILE + (k1 & 15) * C::A3_SBO;
            *reinterpret_cast<float *>(sm + C::OFF_A3H + rb + o_re) = rh;
            *reinterpret_cast<float *>(sm + C::OFF_A3L + rb + o_re) = rl;
            *reinterpret_cast<float *>(sm + C::OFF_A3H + rb + o_im) = ih;
            *reinterpret_cast<float *>(sm + C::OFF_A3L + rb + o_im) = il;
        }
    };
    // P2: D3 -> output tile -> rows of the destination
    auto output = [&](V *dst, int out_cols) {
        const int q = warp & 3;
        const int c = lane & 7;
        if constexpr (C::MT3 == 2) {   // warps of M tile t = (warp / 4) % 2 read k2 in [8 kh, 8 kh + 8)
            const int t = (warp >> 2) & 1, kh = warp >> 3;
            const int k1 = (lane >> 3) + 4 * q + 16 * t;
            float xr[8], xi[8];
            const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + C::D3_COL + t * C::K3 + 8 * kh;
            tc::ld_x8(ta, xr);
            tc::ld_x8(ta + N2, xi);
            tc::wait_ld();
#pragma unroll
            for (int i = 0; i < 8; ++i) outt[(k1 + N1 * (8 * kh + i)) * C::LDO + c] = V{xr[i], xi[i]};
        } else {   // one M tile: warps read k2 in [4 part, 4 part + 4)
            const int part = warp >> 2;
            const int k1 = (lane >> 3) + 4 * q;
            float xr[4], xi[4];
            const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + C::D3_COL + 4 * part;
            tc::ld_x4(ta, xr);
            tc::ld_x4(ta + N2, xi);
            tc::wait_ld();
#pragma unroll
            for (int i = 0; i < 4; ++i) outt[(k1 + N1 * (4 * part + i)) * C::LDO + c] = V{xr[i], xi[i]};
        }
        tc::fence_before_sync();
        __syncthreads();   // output tile complete; D3 read
        const int cc = tid & 7;
        if (cc < out_cols) {
#pragma unroll 4
            for (int k = tid >> 3; k < N; k += C::NT / 8) {
                const int o = orow[k];
                if (o >= 0) dst[o + cc] = outt[k * C::LDO + cc];
            }
        }
        __syncthreads();   // A3's space free again
    };
    // one thread polls (bounded); the block learns the outcome at the barrier
    auto wait_bar = [&](int b, unsigned parity) -> bool {
        bool ok = true;
        if (tid == 0) ok = mbar_wait_bounded(&bar[b], parity, wc.limit);
        return !__syncthreads_or(!ok);
    };

    // ---- the pipeline over units (tile, output)
    bool failed = false;
    unsigned unit = 0;
    bool pend1 = false, pend3 = false;   // step 1 of `unit` / step 3 of `unit - 1` issued and not yet awaited
    V *prev_dst = nullptr;
    int prev_cols = 0;
    load(item);
    while (item < nitems && !failed) {
        int mi, fi, oc, o, c0;
        decode(item, mi, fi, oc, o, c0);
        const double k_out = sp.n_out ? wavenum(o, sp.n_out, sp.dk_out) : 0.0;
        if (sp.mask) {   // rows kept by the dealias mask in column `warp` (< NB): |row index| <= dmax
            if (warp < NB) {
                const double kc = wavenum(c0 + warp, sp.n_col, sp.dk_col);
                int cnt = 0;
                for (int d0 = 0; d0 <= N / 2; d0 += 32) {
                    const int d = d0 + lane;
                    const bool ok = d <= N / 2 && !(ksq3(sp.dk_row * (double)d, k_out, kc) > sp.kmax2);
                    cnt += __popc(__ballot_sync(0xffffffffu, ok));
                }
                if (lane == 0) dmax_s[warp] = cnt - 1;
            }
            __syncthreads();
        }
        const long long dbase = (MB ? mi * sp.ms_out : 0LL) + (long long)(sp.outer_out_compact ? oc : o) * sp.d_out + c0;
        const int out_cols = sp.out_ncols - c0 < NB ? sp.out_ncols - c0 : NB;
        const int nv = sp.nvar[fi];
        const int next = item + gridDim.x;
        for (int v = 0; v < nv; ++v) {
            build_a1(sp.vmul[fi][v], c0, k_out);
            if (v + 1 == nv && next < nitems) load(next);   // the rows of the next tile, in flight meanwhile
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0) issue_step1();
            pend1 = true;
            if (pend3) {   // output of the previous unit while step 1 runs
                if (!wait_bar(1, (unit - 1) & 1u)) { failed = true; break; }
                pend3 = false;
                tc::fence_after_sync();
                output(prev_dst, prev_cols);
            }
            if (!wait_bar(0, unit & 1u)) { failed = true; break; }
            pend1 = false;
            tc::fence_after_sync();
            build_a3();
            fence_proxy_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) issue_step3();
            pend3 = true;
            prev_dst = P.out[sp.vout[fi][v]] + dbase;
            prev_cols = out_cols;
            ++unit;
        }
        item = next;
    }
    if (!failed && pend3) {
        if (wait_bar(1, (unit - 1) & 1u)) {
            pend3 = false;
            tc::fence_after_sync();
            output(prev_dst, prev_cols);
        } else {
            failed = true;
        }
    }
    if (failed) {   // let the MMAs in flight finish (bounded) before the TMEM is freed
        if (tid == 0) {
            if (err) atomicOr(err, 2u);
            if (pend3) mbar_wait_bounded(&bar[1], (unit - 1) & 1u, wc.limit);
            if (pend1) mbar_wait_bounded(&bar[0], unit & 1u, wc.limit);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::dealloc(tmem, C::TCOLS);
    }
}

}  // namespace gnss
