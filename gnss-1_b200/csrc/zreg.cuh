// zreg.cuh -- fused z pass with register-resident line transforms
// (N = 64, 96, 128, 192, 256, 512).
//
// Same work as k_zphys (kz factors and vorticity combinations, C2R of every
// physical quantity of a line pair, the pointwise products, R2C of the
// products), with a different line transform: a warp holds its line in
// registers, E = N/32 elements per lane.  For N = 64 .. 192 (E = 2, 3, 4, 6)
// the transform uses lane shuffles only (zs_fft).  For N = 256, 512 it runs
//   N = E * 32,   32 = E * G   (G = 32/E lanes per group)
//   step A: E-point DFT in registers over elements lane + 32 m, twiddle
//           W_N^(lane k1);
//   one transpose through a padded per-warp scratch;
//   step B: E-point DFT in registers, twiddle W_32^(j k2'), and a G-point
//           DFT across the lanes of a group with shuffles.
// so a line crosses shared memory once per transform (instead of once per
// radix-8 stage).  The C2R packing is done while loading the registers,
// and the twiddles of step A are products of four table powers.  Each warp
// leaves its physical quantity in its own scratch line, where the other warps
// read it; the whole block forms the products in place, into the lines of the
// forward warps.
#pragma once
#include "kernels.cuh"

namespace gnss {

// cos(2 pi e / 32) for e = 0..8; other angles by symmetry.
__host__ __device__ constexpr double cos32_tab(int e) {
    return e == 0   ? 1.0
           : e == 1 ? 0.98078528040323044912618223613424
           : e == 2 ? 0.92387953251128675612818318939679
           : e == 3 ? 0.83146961230254523707878837761791
           : e == 4 ? 0.70710678118654752440084436210485
           : e == 5 ? 0.55557023301960222474283081394853
           : e == 6 ? 0.38268343236508977172845998403040
           : e == 7 ? 0.19509032201612826784828486847702
                    : 0.0;
}
__host__ __device__ constexpr double cos32(int e) {
    e = ((e % 32) + 32) % 32;
    return e <= 8 ? cos32_tab(e) : e <= 16 ? -cos32_tab(16 - e) : e <= 24 ? -cos32_tab(e - 16) : cos32_tab(32 - e);
}
__host__ __device__ constexpr double sin32(int e) { return cos32(e - 8); }

// v * exp(S 2 pi i e / 32) with compile-time e
template <int S, int EXP, typename V> __device__ __forceinline__ V mul_w32(V v) {
    using T = decltype(v.x);
    constexpr int e = ((EXP % 32) + 32) % 32;
    if constexpr (e == 0) {
        return v;
    } else if constexpr (e == 8) {
        return mul_si<S>(v);
    } else if constexpr (e == 16) {
        return V{-v.x, -v.y};
    } else if constexpr (e == 24) {
        return mul_si<-S>(v);
    } else {
        constexpr T c = (T)cos32(e);
        constexpr T s = (T)((double)S * sin32(e));
        return V{v.x * c - v.y * s, v.x * s + v.y * c};
    }
}

// 16-point DFT in natural order: n = 4 n1 + n2, k = k1 + 4 k2.
template <int S, typename V> __device__ __forceinline__ void dft16(V *v) {
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<S>(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
    // v[4 k1 + n2] = y[n2][k1]; twiddle W_16^(n2 k1) = W_32^(2 n2 k1)
    v[5] = mul_w32<S, 2>(v[5]);
    v[9] = mul_w32<S, 4>(v[9]);
    v[13] = mul_w32<S, 6>(v[13]);
    v[6] = mul_w32<S, 4>(v[6]);
    v[10] = mul_w32<S, 8>(v[10]);
    v[14] = mul_w32<S, 12>(v[14]);
    v[7] = mul_w32<S, 6>(v[7]);
    v[11] = mul_w32<S, 12>(v[11]);
    v[15] = mul_w32<S, 18>(v[15]);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<S>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // v[4 k1 + k2] = X[k1 + 4 k2] -> natural order
    V t[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = t[i];
}
template <int S, typename V> struct Dft<16, S, V> {
    static __device__ __forceinline__ void run(V *v) { dft16<S>(v); }
};

// Line lengths the register transforms serve: N = 32 E with E = 8, 16 (one
// transpose through shared memory, zr_fft) or E = 2, 3, 4, 6 (lane shuffles
// only, zs_fft).
__host__ __device__ constexpr bool zr_size(int n) {
    return n == 64 || n == 96 || n == 128 || n == 192 || n == 256 || n == 512;
}

template <typename T, int N> struct ZRCfg {
    static_assert(zr_size(N), "register transforms serve N = 64, 96, 128, 192, 256, 512");
    static constexpr int E = N / 32;                    // elements per lane
    static constexpr bool SHFL = E != 8 && E != 16;     // lane-shuffle scheme (no transpose)
    static constexpr int G = SHFL ? 1 : 32 / E;         // lanes per group in step B (transpose scheme)
    static constexpr int S = 32 + G;                    // transpose row stride (conflict-free both ways)
    // table rows: in the FP32 passes the transpose scheme reads its step-A
    // twiddles W_N^(lane k1) from the table (row k1 - 1, k1 = 1 .. E-1;
    // TWFULL); the z kernels and FP64 build them from the powers
    // W^(lane 2^b), b < LOGE (measured at 512^3 with the full table: FP32
    // passes 0.06 ms faster per step, the z kernel 0.02 ms slower, FP64 0.1 ms
    // slower); the shuffle scheme reads W_N^(lane k1), k1 = 1 .. E-1, then
    // W_32^lane
    static constexpr bool TWFULL = !SHFL && sizeof(T) == 4;
    // rows of the table with (full, where TWFULL) or without the full step-A twiddles; the z kernels use the
    // powers (their shared-memory traffic is the tighter limit), the passes the full table
    __host__ __device__ static constexpr int rows(bool full) {
        return (SHFL || (full && TWFULL)) ? E : (E == 16 ? 4 : 3);
    }
    static constexpr int LOGE = rows(false);
    // line padding.  Transpose scheme: a warp's stores of a transform's
    // output (zr_out_index: lane groups j = lane % G at E^2 sigma(j) apart,
    // lanes of a group on consecutive entries) take one wavefront per 128
    // bytes when every group starts on its own bank range, so PADP entries
    // follow every PADB = E^2: 64 bytes for E = 16 (two groups), 32 for E = 8
    // (four) (measured at 512^3: FP64 z 6.42 -> 6.20 ms, FP32 2.61 -> 2.53 ms;
    // at 256^3 FP64 1.11 -> 0.96 ms).  Shuffle scheme: c entries per E, so
    // that a warp's stores of one output element (positions q + E j,
    // j = 0 .. 31) fall in distinct bank pairs.
    static constexpr int PADB = SHFL ? E : E * E;
    static constexpr int PADP = SHFL ? 0 : (E == 16 ? 64 : 32) / (int)sizeof(V2<T>);
    static constexpr int PADC = SHFL ? ((E & 1) ? 2 : 1) : 0;
    __host__ __device__ static constexpr int pidx(int n) {
        return SHFL ? n + PADC * (n / E) : n + PADP * (n / PADB);
    }
    static constexpr int PL = SHFL ? N + PADC * 32 : N + PADP * (N / PADB);   // line length in shared memory
    static constexpr int SCR = SHFL ? PL : E * S;       // scratch line per warp (transposes, physical line)
    static_assert(SCR >= PL, "scratch holds a padded line");
    // index into the length-N table exp(-2 pi i j / N) of twiddle-table entry i
    __host__ __device__ static constexpr int tw_index(int i, bool full = false) {
        const int row = i >> 5, l = i & 31;
        return SHFL ? (row < E - 1 ? (l * (row + 1)) % N : (E * l) % N)
                    : ((full && TWFULL) ? (l * (row + 1)) % N : (l << row) % N);
    }
    // twiddle powers, scratch lines (one per warp; they also hold the physical
    // lines and the products), raw staging, mbarrier (16 B), kz table (ncp T)
    __host__ __device__ static constexpr int smem_bytes(int nph, int nraw, int ncp) {
        return (LOGE * 32 + nph * SCR + nraw * 2 * ncp) * (int)sizeof(V2<T>) + 16 + ncp * (int)sizeof(T);
    }
    // k_zws: one more scratch line per forward warp
    __host__ __device__ static constexpr int smem_bytes_ws(int nph, int nout, int nraw, int ncp) {
        return smem_bytes(nph + nout, nraw, ncp);
    }
};

// 6-point DFT in natural order: n = 2 n1 + n2, k = k1 + 3 k2 (two 3-point
// DFTs, twiddles W_6^(n2 k1), one 2-point stage).
template <int S, typename V> struct Dft<6, S, V> {
    static __device__ __forceinline__ void run(V *v) {
        using T = decltype(v[0].x);
        const T h = T(0.5);
        const T s3 = T(S) * T(0.86602540378443864676372317075294);
        V a[3] = {v[0], v[2], v[4]}, b[3] = {v[1], v[3], v[5]};
        Dft<3, S, V>::run(a);
        Dft<3, S, V>::run(b);
        b[1] = V{h * b[1].x - s3 * b[1].y, h * b[1].y + s3 * b[1].x};     // W_6^1 = 1/2 + i S sqrt(3)/2
        b[2] = V{-h * b[2].x - s3 * b[2].y, -h * b[2].y + s3 * b[2].x};   // W_6^2 = -1/2 + i S sqrt(3)/2
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
            v[k1] = cadd(a[k1], b[k1]);
            v[k1 + 3] = csub(a[k1], b[k1]);
        }
    }
};

// Output slot of a lane group member after the G-point cross-lane DFT.
template <int G> __device__ __forceinline__ int zr_sigma(int j) {
    return G == 2 ? j : ((j >> 1) | ((j & 1) << 1));
}

// v * W_32^(j Q): lane group member j multiplies, the others keep v
template <int S, int Q, int G, typename V> __device__ __forceinline__ V zr_tw32(V v, int j) {
    using T = decltype(v.x);
    if constexpr (G == 2) {
        if (j) v = mul_w32<S, Q>(v);
        return v;
    } else {
        constexpr T c1 = (T)cos32(Q), s1 = (T)((double)S * sin32(Q));
        constexpr T c2 = (T)cos32(2 * Q), s2 = (T)((double)S * sin32(2 * Q));
        constexpr T c3 = (T)cos32(3 * Q), s3 = (T)((double)S * sin32(3 * Q));
        if (j == 0) return v;
        const T c = j == 1 ? c1 : j == 2 ? c2 : c3;
        const T s = j == 1 ? s1 : j == 2 ? s2 : s3;
        return V{v.x * c - v.y * s, v.x * s + v.y * c};
    }
}
template <int S, int G, int Q, int E, typename V> __device__ __forceinline__ void zr_tw32_all(V *x, int j) {
    if constexpr (Q < E) {
        x[Q] = zr_tw32<S, Q, G>(x[Q], j);
        zr_tw32_all<S, G, Q + 1, E>(x, j);
    }
}

template <typename V> __device__ __forceinline__ V shfl_xor_v(V v, int m) {
    return V{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}

// Transpose layout of zr_fft in a warp's own scratch line: row k1 of 32 + G
// entries (conflict-free both ways).
template <typename T, int N> struct ZrScratch {
    __device__ __forceinline__ int operator()(int k1, int i) const { return k1 * ZRCfg<T, N>::S + i; }
};

// Length-N DFT (N = 32 E, E = 2, 3, 4, 6) of one line held by a warp, with
// lane shuffles only.  On entry x[m] is element lane + 32 m; on return x[q]
// is element q + E bitrev5(lane) of the transform.  n = lane + 32 m,
// k = k1 + E k2: an E-point DFT over m in registers, the twiddle
// W_N^(lane k1), then for every k1 a 32-point DFT across the lanes in five
// radix-2 decimation-in-frequency steps (partner lane ^ h: p + s x with s = +1
// on the lower and -1 on the upper lane, the upper one then multiplied by
// W_{2h}^(lane mod h)).  tws rows: W_N^(lane k1), k1 = 1 .. E-1, then W_32^lane
// (exp(-2 pi i ./.), conjugated for SIGN > 0).
template <typename T, int N, int SIGN>
__device__ __forceinline__ void zs_fft(int lane, V2<T> *x, const V2<T> *tws) {
    using V = V2<T>;
    constexpr int E = N / 32;
    auto tw_at = [&](int i) {
        V t = tws[i];
        if (SIGN > 0) t.y = -t.y;
        return t;
    };
    Dft<E, SIGN, V>::run(x);
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) x[k1] = cmul(x[k1], tw_at(32 * (k1 - 1) + lane));
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool upper = (lane & h) != 0;
        const T sg = upper ? T(-1) : T(1);
        V w = V{T(1), T(0)};
        if (h > 1 && upper) w = tw_at(32 * (E - 1) + (lane & (h - 1)) * (16 / h));
#pragma unroll
        for (int q = 0; q < E; ++q) {
            const V p = shfl_xor_v(x[q], h);
            V t = V{p.x + sg * x[q].x, p.y + sg * x[q].y};
            if (h > 1) t = cmul(t, w);
            x[q] = t;
        }
    }
}

// Length-N DFT of one line held by a warp.  On entry x[m] is element
// lane + 32 m; on return x[q] is element k1 + E q + E^2 zr_sigma(j) of the
// transform, with k1 = lane / G, j = lane % G.  The one transpose goes
// through scr at offsets at(k1, i) (row k1 = 0..E-1, entry i = 0..31);
// tws: the twiddle table of ZRCfg (rows tw_index(., FULLTW)).
template <typename T, int N, int SIGN, class AT = ZrScratch<T, N>, bool FULLTW = false>
__device__ __forceinline__ void zr_fft(int lane, V2<T> *x, V2<T> *scr, const V2<T> *tws, AT at = AT{}) {
    using V = V2<T>;
    using Z = ZRCfg<T, N>;
    constexpr int E = Z::E, G = Z::G;
    if constexpr (Z::SHFL) {   // N = 64, 96, 128, 192: no transpose
        (void)scr;
        (void)at;
        zs_fft<T, N, SIGN>(lane, x, tws);
        return;
    } else {
    Dft<E, SIGN, V>::run(x);
    {
        if constexpr (Z::TWFULL && FULLTW) {   // every W^(lane k1) from the table
#pragma unroll
            for (int k1 = 1; k1 < E; ++k1) {
                V t = tws[32 * (k1 - 1) + lane];
                if (SIGN > 0) t.y = -t.y;
                x[k1] = cmul(x[k1], t);
            }
        } else {
            // W^k1 for k1 = 1, 2, 4 (, 8) from the table, the others as products
            // (w3 = w1 w2, w5 = w1 w4, w6 = w2 w4, w7 = w3 w4, w(8+i) = w(i) w8),
            // each applied as soon as it is formed
            auto tw_at = [&](int b) {
                V t = tws[32 * b + lane];
                if (SIGN > 0) t.y = -t.y;
                return t;
            };
            const V w1 = tw_at(0), w2 = tw_at(1), w4 = tw_at(2);
            const V w3 = cmul(w1, w2);
            if constexpr (E == 16) {
                const V w8 = tw_at(3);
                x[8] = cmul(x[8], w8);
                x[9] = cmul(x[9], cmul(w1, w8));
                x[10] = cmul(x[10], cmul(w2, w8));
                x[11] = cmul(x[11], cmul(w3, w8));
                x[12] = cmul(x[12], cmul(w4, w8));
                x[13] = cmul(x[13], cmul(cmul(w1, w4), w8));
                x[14] = cmul(x[14], cmul(cmul(w2, w4), w8));
                x[15] = cmul(x[15], cmul(cmul(w3, w4), w8));
            }
            x[1] = cmul(x[1], w1);
            x[2] = cmul(x[2], w2);
            x[3] = cmul(x[3], w3);
            x[4] = cmul(x[4], w4);
            x[5] = cmul(x[5], cmul(w1, w4));
            x[6] = cmul(x[6], cmul(w2, w4));
            x[7] = cmul(x[7], cmul(w3, w4));
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) scr[at(k1, lane)] = x[k1];
    __syncwarp();
    const int k1 = lane / G, j = lane % G;
#pragma unroll
    for (int l = 0; l < E; ++l) x[l] = scr[at(k1, G * l + j)];
    __syncwarp();
    Dft<E, SIGN, V>::run(x);
    zr_tw32_all<SIGN, G, 1, E>(x, j);
    // G-point DFT across the group: each radix-2 step is p + s x with s = +1 on
    // the lower and -1 on the upper member (p the partner's value)
    if constexpr (G == 2) {
        const T sg = j == 0 ? T(1) : T(-1);
#pragma unroll
        for (int q = 0; q < E; ++q) {
            const V p = shfl_xor_v(x[q], 1);
            x[q] = V{p.x + sg * x[q].x, p.y + sg * x[q].y};
        }
    } else {
        const int j0 = j & 1, j1 = j >> 1;
        const T s1 = j1 == 0 ? T(1) : T(-1), s0 = j0 == 0 ? T(1) : T(-1);
#pragma unroll
        for (int q = 0; q < E; ++q) {
            const V p = shfl_xor_v(x[q], 2);
            V c = V{p.x + s1 * x[q].x, p.y + s1 * x[q].y};
            if (j0 && j1) c = mul_si<SIGN>(c);
            const V p2 = shfl_xor_v(c, 1);
            x[q] = V{p2.x + s0 * c.x, p2.y + s0 * c.y};
        }
    }
    }
}

// Line index held in x[q] after zr_fft.
template <typename T, int N> __device__ __forceinline__ int zr_out_index(int lane, int q) {
    using Z = ZRCfg<T, N>;
    if constexpr (Z::SHFL)
        return q + Z::E * (int)(__brev((unsigned)lane) >> 27);
    else
        return lane / Z::G + Z::E * q + Z::E * Z::E * zr_sigma<Z::G>(lane % Z::G);
}

// C2R packing (as pack_c2r_combo) straight into the registers of zr_fft:
// x[m] = Z_n, n = lane + 32 m.  keep: bit m set when mode min(n, N - n) is a
// kept kz mode (< nkz); tkz: kz wavenumbers (T) of the kept modes.
template <typename T, int N>
__device__ __forceinline__ void zr_pack(int lane, V2<T> *x, const ZRecipe rc, const V2<T> *a0, const V2<T> *a1,
                                        int ncp, unsigned keep, const T *tkz) {
    using V = V2<T>;
    constexpr int E = ZRCfg<T, N>::E;
    const bool any_kz = rc.ikz[0] || (a1 && rc.ikz[1]);
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int n = lane + 32 * m;
        const bool lo = 2 * n <= N;
        const int k = lo ? n : N - n;
        V z = V{T(0), T(0)};
        if ((keep >> m) & 1u) {
            const T kz = any_kz ? tkz[k] : T(0);
            V a = a0[k], b = a0[ncp + k];
            if (rc.ikz[0]) { a = V{-kz * a.y, kz * a.x}; b = V{-kz * b.y, kz * b.x}; }
            if (rc.sgn[0] < 0) { a = V{-a.x, -a.y}; b = V{-b.x, -b.y}; }
            if (a1) {
                V c = a1[k], d = a1[ncp + k];
                if (rc.ikz[1]) { c = V{-kz * c.y, kz * c.x}; d = V{-kz * d.y, kz * d.x}; }
                if (rc.sgn[1] < 0) { a = csub(a, c); b = csub(b, d); }
                else { a = cadd(a, c); b = cadd(b, d); }
            }
            if (k == 0 || 2 * k == N) { a.y = T(0); b.y = T(0); }
            z = lo ? V{a.x - b.y, a.y + b.x} : V{a.x + b.y, b.x - a.y};
        }
        x[m] = z;
    }
}

// The same packing with the recipe fixed at compile time, for the recipes the
// step uses: sgn[0] = +1 and, with a second term, sgn[1] = -1 (IKZ0, IKZ1:
// the kz factor on the first, second term; HAS1: a second term).  Same
// arithmetic as zr_pack in the same order; the keep test is k < nkz, and
// elements of which no lane is kept are skipped by a warp-uniform test.  The
// imaginary parts are cleared only where they can be nonzero modes k = 0 and
// k = N/2, i.e. lane 0 of elements 0 and E/2 (element E/2 uses the upper-half
// formula at lane 0, which gives the same value once they are cleared).
template <typename T, int N, bool IKZ0, bool HAS1, bool IKZ1>
__device__ __forceinline__ void zr_pack_fixed(int lane, V2<T> *x, const V2<T> *a0, const V2<T> *a1, int ncp, int nkz,
                                              const T *tkz) {
    using V = V2<T>;
    constexpr int E = ZRCfg<T, N>::E;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const bool lo = m < E / 2;
        const int kmin = lo ? 32 * m : N - 31 - 32 * m;   // smallest k of the element over the warp
        V z = V{T(0), T(0)};
        if (kmin < nkz) {
            const int k = lo ? lane + 32 * m : N - lane - 32 * m;
            if (k < nkz) {
                V a = a0[k], b = a0[ncp + k];
                T kz = T(0);
                if constexpr (IKZ0 || IKZ1) kz = tkz[k];
                if constexpr (IKZ0) { a = V{-kz * a.y, kz * a.x}; b = V{-kz * b.y, kz * b.x}; }
                if constexpr (HAS1) {
                    V c = a1[k], d = a1[ncp + k];
                    if constexpr (IKZ1) { c = V{-kz * c.y, kz * c.x}; d = V{-kz * d.y, kz * d.x}; }
                    a = csub(a, c);
                    b = csub(b, d);
                }
                if (m == 0 || m == E / 2) {
                    if (lane == 0) { a.y = T(0); b.y = T(0); }
                }
                z = lo ? V{a.x - b.y, a.y + b.x} : V{a.x + b.y, b.x - a.y};
            }
        }
        x[m] = z;
    }
}

// Recipe class for zr_pack_fixed (0 .. 5), or -1 for the general zr_pack.
__device__ __forceinline__ int zr_kind(const ZRecipe &rc) {
    if (rc.sgn[0] != 1) return -1;
    if (rc.r[1] < 0) return rc.ikz[0] ? 1 : 0;
    if (rc.sgn[1] != -1) return -1;
    return 2 + (rc.ikz[0] ? 2 : 0) + (rc.ikz[1] ? 1 : 0);
}

// Packs quantity `rc` of the staged raw line pairs into x (kind = zr_kind(rc)).
template <typename T, int N>
__device__ __forceinline__ void zr_pack_any(int kind, int lane, V2<T> *x, const ZRecipe rc, const V2<T> *raw, int rawf,
                                            int ncp, int nkz, unsigned keep, const T *tkz) {
    const V2<T> *a0 = raw + rc.r[0] * rawf;
    const V2<T> *a1 = rc.r[1] >= 0 ? raw + rc.r[1] * rawf : nullptr;
    switch (kind) {
        case 0: zr_pack_fixed<T, N, false, false, false>(lane, x, a0, a1, ncp, nkz, tkz); break;
        case 1: zr_pack_fixed<T, N, true, false, false>(lane, x, a0, a1, ncp, nkz, tkz); break;
        case 2: zr_pack_fixed<T, N, false, true, false>(lane, x, a0, a1, ncp, nkz, tkz); break;
        case 3: zr_pack_fixed<T, N, false, true, true>(lane, x, a0, a1, ncp, nkz, tkz); break;
        case 4: zr_pack_fixed<T, N, true, true, false>(lane, x, a0, a1, ncp, nkz, tkz); break;
        case 5: zr_pack_fixed<T, N, true, true, true>(lane, x, a0, a1, ncp, nkz, tkz); break;
        default: zr_pack<T, N>(lane, x, rc, a0, a1, ncp, keep, tkz); break;
    }
}

// Pointwise products of one line pair by the whole block: the physical
// quantities are element pidx(n) of the lines `phys` (stride SCR), product f
// goes to element pidx(n) of line f of `out` (stride SCR).  out may equal
// phys (products in place over quantities 0 .. 4): each point is read in full
// by one thread before that thread writes it, quantities 0 .. 4 are read
// before any product is written, and products go to lines 0 .. 4 only.
// Quantities: 0 u, 1 v, 2 w, 3 w1, 4 w2, 5 w3,
// 6 sx, 7 sy, 8 sz, [9 cx, 10 cy, 11 cz], [12 c, 13 lap s]; products as
// zphys_products: (w x u) (crossProductKernel_mgpu, solver.cu:139-164),
// u . grad s (dotKernel_mgpu, solver.cu:342-356) and the colloid term
// (colloidAdvectionKernel_mgpu, solver.cu:374-388).
// With DIAG, the thread also adds to acc the vorticity sums of its points
// (ZR_VORT_SUMS: |w|, w_x^2, w_y^2, w_z^2, both lines of the pair), the sums
// of k_vort_partial (statistics.cu:1211-1305), from the physical quantities 3,
// 4, 5 = w_x, w_y, w_z it reads anyway.
constexpr int ZR_VORT_SUMS = 4;
template <typename T, int N, int NPH, bool DIAG = false>
__device__ __forceinline__ void zr_products(const V2<T> *phys, V2<T> *out, T alpha, double *acc = nullptr) {
    using V = V2<T>;
    using Z = ZRCfg<T, N>;
    constexpr int SCR = Z::SCR;
    constexpr bool has_c = NPH >= 12, has_al = NPH >= 14;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        const int pn = Z::pidx(n);
        const V *p = phys + pn;
        const V u = p[0 * SCR], v = p[1 * SCR], w = p[2 * SCR];
        const V o1 = p[3 * SCR], o2 = p[4 * SCR], o3 = p[5 * SCR];
        const V sx = p[6 * SCR], sy = p[7 * SCR], sz = p[8 * SCR];
        if constexpr (DIAG) {
            const double ax = o1.x, ay = o2.x, az = o3.x, bx = o1.y, by = o2.y, bz = o3.y;
            acc[0] += sqrt(ax * ax + ay * ay + az * az) + sqrt(bx * bx + by * by + bz * bz);
            acc[1] += ax * ax + bx * bx;
            acc[2] += ay * ay + by * by;
            acc[3] += az * az + bz * bz;
        }
        V *o = out + pn;
        o[0 * SCR] = V{o2.x * w.x - o3.x * v.x, o2.y * w.y - o3.y * v.y};
        o[1 * SCR] = V{-o1.x * w.x + o3.x * u.x, -o1.y * w.y + o3.y * u.y};
        o[2 * SCR] = V{o1.x * v.x - o2.x * u.x, o1.y * v.y - o2.y * u.y};
        o[3 * SCR] = V{u.x * sx.x + v.x * sy.x + w.x * sz.x, u.y * sx.y + v.y * sy.y + w.y * sz.y};
        if constexpr (has_c) {
            const V cx = p[9 * SCR], cy = p[10 * SCR], cz = p[11 * SCR];
            const V adv = V{u.x * cx.x + v.x * cy.x + w.x * cz.x, u.y * cx.y + v.y * cy.y + w.y * cz.y};
            if constexpr (has_al) {
                const V cc = p[12 * SCR], ls = p[13 * SCR];
                const V dr = V{ls.x * cc.x + cx.x * sx.x + cy.x * sy.x + cz.x * sz.x,
                               ls.y * cc.y + cx.y * sx.y + cy.y * sy.y + cz.y * sz.y};
                o[4 * SCR] = V{alpha * dr.x + adv.x, alpha * dr.y + adv.y};
            } else {
                o[4 * SCR] = adv;
            }
        }
    }
}

// R2C output of one product line: the length-N transform in x (element
// zr_out_index(lane, q) in x[q]) goes through the warp's scratch line, and the
// kept modes of the two real lines of the pair are stored as the raw layout
// ([A: ncp][B: ncp]) at d.
template <typename T, int N>
__device__ __forceinline__ void zr_store_r2c(int lane, const V2<T> *x, V2<T> *scr, V2<T> *d, int ncp) {
    using V = V2<T>;
    using Z = ZRCfg<T, N>;
#pragma unroll
    for (int q = 0; q < Z::E; ++q) scr[Z::pidx(zr_out_index<T, N>(lane, q))] = x[q];
    __syncwarp();
    for (int k = lane; k < ncp; k += 32) {
        V A = V{T(0), T(0)}, B = V{T(0), T(0)};
        if (2 * k <= N) {
            const V zk = scr[Z::pidx(k)];
            const V zm = scr[Z::pidx((N - k) % N)];
            A = V{T(0.5) * (zk.x + zm.x), T(0.5) * (zk.y - zm.y)};
            B = V{T(0.5) * (zk.y + zm.y), T(-0.5) * (zk.x - zm.x)};
        }
        d[k] = A;
        d[ncp + k] = B;
    }
    __syncwarp();   // scratch reused by the next transform
}

// Persistent: block b handles line pairs b, b + gridDim.x, ... of all members
// of a batch (npairs in all, mpairs per member, members ms elements apart);
// warp q forms physical quantity q.  The raw lines of the next pair arrive by
// cp.async.bulk (CTA-local, no multicast) while the current pair is
// processed; a wait that times out sets bit 0 of *err and the block stops.
// With DIAG the block also writes one row of ZR_VORT_SUMS vorticity sums over
// its points to diag[blockIdx.x] (fixed-order reduction), for the statistics
// of the state the step starts from.
template <typename T, int N, int NPH, int NRAW, bool DIAG = false, bool MB = false>
__global__ void __launch_bounds__(NPH * 32, (sizeof(T) == 4 && NPH <= 9) ? (N <= 192 ? 4 : 3) : (N <= 192 ? 2 : 1))
k_zreg(const __grid_constant__ FieldSet<T> f, const __grid_constant__ ZRecipeSet zr, int nout, long long npairs,
       int ncp, int nkz, T scale, T alpha, double dkz, const V2<T> *__restrict__ tw, unsigned *__restrict__ err,
       double *__restrict__ diag, long long mpairs, long long ms) {
    using V = V2<T>;
    using Z = ZRCfg<T, N>;
    constexpr int E = Z::E, SCR = Z::SCR;
    double acc[DIAG ? ZR_VORT_SUMS : 1] = {};
    const int rawf = 2 * ncp;
    const unsigned raw_bytes = (unsigned)(rawf * sizeof(V));
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    V *scr_all = tws + Z::LOGE * 32;
    V *raw = scr_all + NPH * SCR;
    uint64_t *bar = reinterpret_cast<uint64_t *>(raw + NRAW * rawf);
    T *tkz = reinterpret_cast<T *>(bar + 2);   // kz wavenumbers of the kept modes (ncp entries)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    long long pair = blockIdx.x;
    if (pair >= npairs) return;   // uniform for the block
    for (int i = threadIdx.x; i < Z::LOGE * 32; i += blockDim.x) tws[i] = tw[Z::tw_index(i)];
    for (int k = threadIdx.x; k < ncp; k += blockDim.x) tkz[k] = (T)wavenum(k, N, dkz);
    unsigned keep = 0;   // bit m: mode min(n, N - n) of element n = lane + 32 m is kept
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int n = (threadIdx.x & 31) + 32 * m;
        keep |= ((2 * n <= N ? n : N - n) < nkz ? 1u : 0u) << m;
    }
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    pdl_wait();
    const WaitCtl wc(err);
    auto issue = [&](long long p, bool withhold = false) {
        mbar_arrive_expect_tx(bar, NRAW * raw_bytes);
        if (!withhold)
            for (int q = 0; q < NRAW; ++q) bulk_g2s(raw + q * rawf, f.p[q] + pair_offset<MB>(p, mpairs, ms, rawf), raw_bytes, bar);
    };
    if (threadIdx.x == 0) issue(pair, wc.withhold);
    unsigned parity = 0;
    const ZRecipe rc = zr.q[warp];
    const int kind = zr_kind(rc);
    V *scr = scr_all + warp * SCR;   // transposes, then this warp's physical quantity
    for (; pair < npairs; pair += gridDim.x) {
        const bool ok = mbar_wait_bounded(bar, parity, wc.limit);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(err, 1u);
            mbar_wait_bounded(bar, parity, wc.limit);   // let an overdue copy land before leaving
            return;
        }
        parity ^= 1u;
        V x[E];
        if constexpr (sizeof(T) == 8 && E % 2 == 0)   // measured: faster in FP64; in FP32 the general form keeps 72 registers
            zr_pack_any<T, N>(kind, lane, x, rc, raw, rawf, ncp, nkz, keep, tkz);
        else
            zr_pack<T, N>(lane, x, rc, raw + rc.r[0] * rawf, rc.r[1] >= 0 ? raw + rc.r[1] * rawf : nullptr, ncp, keep,
                          tkz);
        __syncthreads();   // staging consumed; the previous pair's products are read
        if (threadIdx.x == 0 && pair + gridDim.x < npairs) {
            fence_proxy_async_smem();
            issue(pair + gridDim.x);
        }
        zr_fft<T, N, +1>(lane, x, scr, tws);   // ends its scratch reads with __syncwarp
#pragma unroll
        for (int q = 0; q < E; ++q) scr[Z::pidx(zr_out_index<T, N>(lane, q))] = cscale(x[q], scale);
        __syncthreads();   // every physical quantity on chip
        zr_products<T, N, NPH, DIAG>(scr_all, scr_all, alpha, acc);
        __syncthreads();   // products in the scratch lines of warps 0 .. nout-1
        if (warp < nout) {   // z R2C of product `warp`, written over raw field `warp` of the pair
#pragma unroll
            for (int m = 0; m < E; ++m) x[m] = scr[Z::pidx(lane + 32 * m)];
            __syncwarp();
            zr_fft<T, N, -1>(lane, x, scr, tws);
            zr_store_r2c<T, N>(lane, x, scr, f.p[warp] + pair_offset<MB>(pair, mpairs, ms, rawf), ncp);
        }
    }
    if constexpr (DIAG) {   // warp shuffles, then the block's warps in order
        __shared__ double red[ZR_VORT_SUMS][NPH];
#pragma unroll
        for (int q = 0; q < ZR_VORT_SUMS; ++q) {
            double v = acc[q];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[q][warp] = v;
        }
        __syncthreads();
        if (threadIdx.x < ZR_VORT_SUMS) {
            double v = 0.0;
            for (int w = 0; w < NPH; ++w) v += red[threadIdx.x][w];
            diag[blockIdx.x * ZR_VORT_SUMS + threadIdx.x] = v;
        }
    }
}

// Warp-specialised form of k_zreg (same arguments, same results): NPH inverse
// warps and nout forward warps per block, each with its own scratch line.
// Per line pair p, between two block barriers, the inverse warps unpack and
// transform the quantities of p (each leaving its physical quantity in its
// own line) while the forward warps transform and store the products of the
// block's previous pair (held in their own lines); after the first barrier
// the whole block forms the products of p into the forward warps' lines.
// Every warp thus runs one length-N transform per pair instead of nout of
// NPH warps running the forward ones alone.  The raw lines of the next pair
// are requested as soon as every inverse warp has unpacked (named barrier 1);
// a wait that times out sets bit 0 of *err and the block stops.  FP32 with 9
// quantities: 13 warps, 72 registers, two blocks per SM; FP64 with 9 or 12
// quantities: 13 or 17 warps, one block per SM (k_zreg: 9 or 12).
template <int NPH> __host__ __device__ constexpr int zws_nout() { return NPH >= 12 ? 5 : 4; }
template <typename T, int N, int NPH, int NRAW, bool MB = false>
__global__ void __launch_bounds__((NPH + zws_nout<NPH>()) * 32, sizeof(T) == 4 ? 2 : 1)
k_zws(const __grid_constant__ FieldSet<T> f, const __grid_constant__ ZRecipeSet zr, int nout, long long npairs,
      int ncp, int nkz, T scale, T alpha, double dkz, const V2<T> *__restrict__ tw, unsigned *__restrict__ err,
      long long mpairs, long long ms) {
    constexpr int NOUT = zws_nout<NPH>();   // products (the host checks nout)
    static_assert(NPH == 9 || NPH == 12, "k_zws serves 9 or 12 physical quantities");
    using V = V2<T>;
    using Z = ZRCfg<T, N>;
    constexpr int E = Z::E, SCR = Z::SCR;
    constexpr unsigned NINV = NPH * 32;   // threads of the inverse warps (named barrier 1)
    (void)nout;
    const int rawf = 2 * ncp;
    const unsigned raw_bytes = (unsigned)(rawf * sizeof(V));
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    V *lines = tws + Z::LOGE * 32;           // NPH + NOUT scratch lines, one per warp
    V *raw = lines + (NPH + NOUT) * SCR;
    uint64_t *bar = reinterpret_cast<uint64_t *>(raw + NRAW * rawf);
    T *tkz = reinterpret_cast<T *>(bar + 2);   // kz wavenumbers of the kept modes (ncp entries)
    __shared__ int stop;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    long long pair = blockIdx.x;
    if (pair >= npairs) return;   // uniform for the block
    for (int i = threadIdx.x; i < Z::LOGE * 32; i += blockDim.x) tws[i] = tw[Z::tw_index(i)];
    for (int k = threadIdx.x; k < ncp; k += blockDim.x) tkz[k] = (T)wavenum(k, N, dkz);
    unsigned keep = 0;   // bit m: mode min(n, N - n) of element n = lane + 32 m is kept
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int n = lane + 32 * m;
        keep |= ((2 * n <= N ? n : N - n) < nkz ? 1u : 0u) << m;
    }
    if (threadIdx.x == 0) {
        stop = 0;
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    pdl_wait();
    const WaitCtl wc(err);
    auto issue = [&](long long p, bool withhold = false) {
        mbar_arrive_expect_tx(bar, NRAW * raw_bytes);
        if (!withhold)
            for (int q = 0; q < NRAW; ++q) bulk_g2s(raw + q * rawf, f.p[q] + pair_offset<MB>(p, mpairs, ms, rawf), raw_bytes, bar);
    };
    if (threadIdx.x == 0) issue(pair, wc.withhold);
    unsigned parity = 0;
    const bool inv = warp < NPH;
    const ZRecipe rc = zr.q[inv ? warp : 0];
    const int kind = zr_kind(rc);
    V *scr = lines + warp * SCR;
    long long prev = -1;
    for (;;) {
        if (inv) {
            if (pair < npairs) {
                const bool ok = mbar_wait_bounded(bar, parity, wc.limit);
                V x[E];
                if constexpr (sizeof(T) == 8 && E % 2 == 0)   // as k_zreg
                    zr_pack_any<T, N>(kind, lane, x, rc, raw, rawf, ncp, nkz, keep, tkz);
                else
                    zr_pack<T, N>(lane, x, rc, raw + rc.r[0] * rawf, rc.r[1] >= 0 ? raw + rc.r[1] * rawf : nullptr,
                                  ncp, keep, tkz);
                if (bar_named_or(1, NINV, !ok)) {   // every inverse warp has unpacked, or one gave up
                    if (threadIdx.x == 0) {
                        stop = 1;
                        mbar_wait_bounded(bar, parity, wc.limit);   // let an overdue copy land before leaving
                    }
                } else {
                    parity ^= 1u;
                    if (threadIdx.x == 0 && pair + gridDim.x < npairs) {
                        fence_proxy_async_smem();
                        issue(pair + gridDim.x);
                    }
                    zr_fft<T, N, +1>(lane, x, scr, tws);   // ends its scratch reads with __syncwarp
#pragma unroll
                    for (int q = 0; q < E; ++q) scr[Z::pidx(zr_out_index<T, N>(lane, q))] = cscale(x[q], scale);
                }
            }
        } else if (prev >= 0) {   // z R2C of product warp - NPH of the previous pair
            V x[E];
#pragma unroll
            for (int m = 0; m < E; ++m) x[m] = scr[Z::pidx(lane + 32 * m)];
            __syncwarp();
            zr_fft<T, N, -1>(lane, x, scr, tws);
            zr_store_r2c<T, N>(lane, x, scr, f.p[warp - NPH] + pair_offset<MB>(prev, mpairs, ms, rawf), ncp);
        }
        __syncthreads();   // quantities of `pair` in the inverse warps' lines; the forward lines are free
        if (stop) {
            if (threadIdx.x == 0) atomicOr(err, 1u);
            return;
        }
        if (pair >= npairs) break;
        zr_products<T, N, NPH>(lines, lines + NPH * SCR, alpha);
        __syncthreads();   // products of `pair` in the forward warps' lines
        prev = pair;
        pair += gridDim.x;
    }
}

}  // namespace gnss
