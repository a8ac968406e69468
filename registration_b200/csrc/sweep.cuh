// Generic tiled N-body sweep over (target block, source chunk) items.
//
// Each block owns BLOCK*R targets (R per thread, kept in registers) and one
// chunk of the source range.  Source records (NS 16-byte words each, packed
// structure-of-arrays in global memory, see Op::Src) are streamed through
// shared memory in tiles of TILE records with a two-stage cp.async pipeline;
// every warp reads the same record at the same time (shared-memory broadcast).
// Per-target accumulators: FP32 partials over FOLD sources, folded into a
// TwoSum-compensated (sum, err) pair (FP32 ops), or plain FP64 sums.
// The block writes its per-target sums as doubles into the partial buffer
//   part[(seg.part + chunk * seg.n_tgt + t) * Op::NOUT + c]
// and a separate combine kernel adds the chunks in a fixed order, so results
// do not depend on scheduling.
//
// SYM (symmetric sums, used for energies <S,S> - 2 <S,T> whose summand is
// symmetric in the target and the source): the first seg.sym_tiles source
// tiles hold the targets' own records in target order.  A target block skips
// those of its own records that precede it, counts its diagonal tiles once
// and the later ones twice (per-tile weight applied to the FP32 fold partial,
// exact for 1 and 2), so each unordered pair is evaluated once: the per-target
// partial sums are no longer the per-target sums, their weighted total is.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace lddmm {

// An operator may accumulate some outputs scaled by a power of two (cheaper per
// pair); Op::out_scale(c) is then the exact factor applied when they are written.
template <class Op, class = void>
struct op_has_out_scale : std::false_type {};
template <class Op>
struct op_has_out_scale<Op, std::void_t<decltype(Op::out_scale(0))>> : std::true_type {};

// An operator may ask for a minimum number of resident blocks per SM
// (Op::MIN_BLOCKS), which caps its registers per thread.
template <class Op, class = void>
struct op_min_blocks : std::integral_constant<int, 1> {};
template <class Op>
struct op_min_blocks<Op, std::void_t<decltype(Op::MIN_BLOCKS)>> : std::integral_constant<int, Op::MIN_BLOCKS> {};

template <class Op, bool SYM = false>
__global__ void __launch_bounds__(Op::BLOCK, op_min_blocks<Op>::value) sweep_kernel(const SweepGrid grid, const typename Op::Params P,
                                                           double* __restrict__ part) {
    using Real = typename Op::Real;
    constexpr int BLOCK = Op::BLOCK, R = Op::R, TILE = Op::TILE, NS = Op::NS, NOUT = Op::NOUT;
    constexpr int WORDS_PER_REC = NS;                  // 16-byte words per source record
    constexpr int WORDS_PER_TILE = WORDS_PER_REC * TILE;
    static_assert(WORDS_PER_TILE % BLOCK == 0, "tile must split evenly over the block");
    __shared__ __align__(16) float4 smem[2][WORDS_PER_TILE];

    const int item = blockIdx.x;
    const SegDesc sg = find_segment(grid, item);
    const int local = item - sg.item0;
    const int tb = local % sg.n_tb;
    const int chunk = local / sg.n_tb;
    int tile_lo = (int)(((long long)chunk * sg.n_src_tiles) / sg.split);
    const int tile_hi = (int)(((long long)(chunk + 1) * sg.n_src_tiles) / sg.split);
    int diag_hi = 0;   // SYM: own tiles at or after diag_hi (and before sym_tiles) count twice
    if constexpr (SYM) {
        static_assert((BLOCK * R) % TILE == 0, "symmetric sweeps need whole tiles per target block");
        constexpr int TPB = (BLOCK * R) / TILE;
        const int diag_lo = tb * TPB < sg.sym_tiles ? tb * TPB : sg.sym_tiles;
        diag_hi = tb * TPB + TPB;
        if (tile_lo < diag_lo) tile_lo = diag_lo < tile_hi ? diag_lo : tile_hi;
    }

    // targets owned by this thread: t = tb*BLOCK*R + r*BLOCK + threadIdx.x (rows are padded);
    // an operator with TPS == 2 keeps two of them per slot (packed FP32 pairs)
    constexpr int TPS = Op::TPS;
    constexpr int SLOTS = R / TPS;
    static_assert(R % TPS == 0, "R must be a multiple of TPS");
    typename Op::Tgt tg[SLOTS];
#pragma unroll
    for (int q = 0; q < SLOTS; ++q) {
        const long long row = sg.tgt + (long long)tb * BLOCK * R + (q * TPS) * BLOCK + threadIdx.x;
        if constexpr (TPS == 1) Op::load_target(P, row, tg[q]);
        else Op::load_target(P, row, row + BLOCK, tg[q]);
    }
    typename Op::Acc acc[SLOTS];
#pragma unroll
    for (int q = 0; q < SLOTS; ++q) acc[q].zero();

    // global source words: Op lays a record out as NS planes of float4 words,
    // plane p of record j at P.src4[p * P.src_stride + j]
    auto load_tile = [&](int tile, int stage) {
        const long long rec0 = sg.src + (long long)tile * TILE;
#pragma unroll
        for (int w = threadIdx.x; w < WORDS_PER_TILE; w += BLOCK) {
            const int plane = w / TILE;
            const int j = w - plane * TILE;
            cp_async16(&smem[stage][w], P.src4 + (long long)plane * P.src_stride + rec0 + j);
        }
        cp_async_commit();
    };

    if (tile_lo < tile_hi) load_tile(tile_lo, 0);
    for (int tile = tile_lo; tile < tile_hi; ++tile) {
        const int stage = (tile - tile_lo) & 1;
        if (tile + 1 < tile_hi) {
            load_tile(tile + 1, stage ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float4* S = smem[stage];
        const float wt = (SYM && tile >= diag_hi && tile < sg.sym_tiles) ? 2.f : 1.f;
        (void)wt;
#pragma unroll 1
        for (int j0 = 0; j0 < TILE; j0 += Op::FOLD) {
#pragma unroll
            for (int q = 0; q < SLOTS; ++q) acc[q].begin_fold();
#pragma unroll 4
            for (int j = j0; j < j0 + Op::FOLD; ++j) {
                typename Op::Src s;
                Op::load_source(S, j, s);
#pragma unroll
                for (int q = 0; q < SLOTS; ++q) Op::pair(P, tg[q], s, acc[q]);
            }
#pragma unroll
            for (int q = 0; q < SLOTS; ++q) {
                if constexpr (SYM) acc[q].end_fold_w(wt);
                else acc[q].end_fold();
            }
        }
        __syncthreads();
    }

#pragma unroll
    for (int q = 0; q < SLOTS; ++q) {
#pragma unroll
        for (int lane = 0; lane < TPS; ++lane) {
            const int t = tb * BLOCK * R + (q * TPS + lane) * BLOCK + threadIdx.x;
            if (t < sg.n_tgt) {
                double* dst = part + (sg.part + (long long)chunk * sg.n_tgt + t) * NOUT;
#pragma unroll
                for (int c = 0; c < NOUT; ++c) {
                    double v;
                    if constexpr (TPS == 1) v = acc[q].value(c);
                    else v = acc[q].value(c, lane);
                    if constexpr (op_has_out_scale<Op>::value) v *= Op::out_scale(c);
                    dst[c] = v;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Accumulators
// ---------------------------------------------------------------------------
// FP32 partial over FOLD sources + TwoSum-compensated running sum.
template <int N>
struct AccF32C {
    float p[N], s[N], e[N];
    LDDMM_D void zero() {
#pragma unroll
        for (int c = 0; c < N; ++c) s[c] = e[c] = 0.f;
    }
    LDDMM_D void begin_fold() {
#pragma unroll
        for (int c = 0; c < N; ++c) p[c] = 0.f;
    }
    LDDMM_D void end_fold() {
#pragma unroll
        for (int c = 0; c < N; ++c) two_sum_acc(s[c], e[c], p[c]);
    }
    LDDMM_D void end_fold_w(float w) {
#pragma unroll
        for (int c = 0; c < N; ++c) two_sum_acc(s[c], e[c], p[c] * w);
    }
    LDDMM_D void add(int c, float v) { p[c] += v; }
    LDDMM_D void fma(int c, float a, float b) { p[c] = fmaf(a, b, p[c]); }
    LDDMM_D double value(int c) const { return (double)s[c] + (double)e[c]; }
};

// Plain FP64 accumulation (the uncompensated FP64 comparator path).
template <int N>
struct AccF64 {
    double s[N];
    LDDMM_D void zero() {
#pragma unroll
        for (int c = 0; c < N; ++c) s[c] = 0.0;
    }
    double m[N];   // running sum at the start of the fold (symmetric sweeps)
    LDDMM_D void begin_fold() {
#pragma unroll
        for (int c = 0; c < N; ++c) m[c] = s[c];
    }
    LDDMM_D void end_fold() {}
    LDDMM_D void end_fold_w(float w) {
        if (w != 1.f)
#pragma unroll
            for (int c = 0; c < N; ++c) s[c] = m[c] + (double)w * (s[c] - m[c]);
    }
    LDDMM_D void add(int c, double v) { s[c] += v; }
    LDDMM_D void fma(int c, double a, double b) { s[c] = fma_rn(a, b, s[c]); }
    LDDMM_D double value(int c) const { return s[c]; }
    static LDDMM_D double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
};

}  // namespace lddmm
