// Host-side check of the shared-memory and tensor-copy geometry of the fragment kernel (n = 8)
// and of the generic stage kernel's TMA and paired-row TMA forms, for every compiled order and both precisions: box
// widths within the
// tensor-copy limit and 16-byte multiples, every staged array on a 128-byte boundary, the stage
// ring within the shared memory of one CTA.  Prints one line per failure and "ALL OK" otherwise.
#include <cstdio>

#include "vlasov_stage_frag.cuh"
#include "vlasov_stage_gen.cuh"

static int failures = 0;

static void expect(bool ok, const char *what, int n, int es) {
    if (!ok) {
        std::printf("FAIL n=%d element=%dB: %s\n", n, es, what);
        ++failures;
    }
}

template <int N, typename T>
void check_tma() {
    using G = vl::GenTmaGeom<N, T>;
    const int es = (int)sizeof(T);
    expect(G::WB % G::Q == 0, "TMA row width is a whole number of 16-byte units", N, es);
    expect(G::WB <= 256, "TMA box width <= 256 elements", N, es);
    expect((G::WB * sizeof(T)) % 16 == 0, "TMA box inner extent is a 16-byte multiple", N, es);
    expect(G::RJ >= N, "rows per plane cover the j extent", N, es);
    expect(G::WB >= G::EPT * N + 2 + (G::Q - 1), "row holds the tile, both traces and the alignment offset", N, es);
    expect(G::IN_B % 128 == 0 && G::FN_B % 128 == 0 && G::FSIDE_B % 128 == 0 && G::XF_B % 128 == 0 &&
               G::UF_B % 128 == 0 && G::BGSIDE_B % 128 == 0 && G::UX_B % 128 == 0 && G::STAGE_B % 128 == 0,
           "every staged array starts on a 128-byte boundary", N, es);
    expect(G::UX_B >= sizeof(double) * (size_t)G::UXC, "u-node slot holds the even-aligned copy", N, es);
    expect(G::smem_bytes() <= 227 * 1024, "stage ring fits the shared memory of one CTA", N, es);
}

// paired-row TMA form (FP32 rows of R = 2 mod 4 floats): staged arrays, box extents, and for a
// range of grids the box coordinates the kernel issues (every tile of every u and v element): the
// innermost coordinate a 16-byte multiple, each parity's used columns (left trace .. right trace)
// inside its own row of the pair and inside the box, every row of the tile inside the box's pairs,
// the u-trace rows inside the state
template <int N>
void check_pair() {
    using G = vl::GenPairGeom<N, float>;
    const int es = 4;
    expect(G::WB % G::Q == 0 && G::WB <= 256, "paired box width: 16-byte units, <= 256", N, es);
    expect(G::NPJ <= 256 && 2 * G::NPJ >= N + 1, "row pairs span the n rows at either parity", N, es);
    expect(G::BLK % 128 == 0 && G::IN_B % 128 == 0 && G::FPB % 128 == 0 && G::XF_B % 128 == 0 &&
               G::FSIDE_B % 128 == 0 && G::UF_B % 128 == 0 && G::BG_B % 128 == 0 && G::UX_B % 128 == 0 &&
               G::STAGE_B % 128 == 0,
           "every paired-form array starts on a 128-byte boundary", N, es);
    expect(G::smem_bytes() <= 227 * 1024, "paired stage ring fits the shared memory of one CTA", N, es);
    constexpr int EPT = G::EPT, Q = G::Q;
    for (int nu = 1; nu <= 12; ++nu) {
        for (int nv = 1; nv <= 70; ++nv) {
            const long U = nu + 2, V = nv + 2, R = V * N;
            if (R % 4 != 2 || (U * N) % 2 != 0) continue;
            const int nbt = (nv + EPT - 1) / EPT;
            for (int au = 0; au < nu; ++au) {
                const long Ag = au + 1, r0 = Ag * N, p0 = r0 / 2;
                for (int bt = 0; bt < nbt; ++bt) {
                    const int b0 = bt * EPT, nb = (nv - b0) < EPT ? (nv - b0) : EPT;
                    const long cL = (long)(b0 + 1) * N - 1;
                    for (int par = 0; par < 2; ++par) {
                        const long cp = par * R + cL;          // left trace column in the pair
                        const long xs = cp & ~(long)(Q - 1);   // box start
                        expect(xs % Q == 0 && xs >= 0, "paired box x coordinate is a 16-byte multiple", N, es);
                        const long lo = cp, hi = cp + 1 + (long)nb * N;   // left .. right trace
                        expect(lo >= par * R && hi < (par + 1) * R, "parity's columns inside its own row", N, es);
                        expect(hi - xs < G::WB, "parity's columns inside the box", N, es);
                    }
                    for (int j = 0; j < N; ++j) {
                        const long idx = (r0 + j) / 2 - p0;
                        expect(idx >= 0 && idx < G::NPJ, "tile row inside the box's pairs", N, es);
                    }
                    expect(p0 + G::NPJ <= U * N / 2 + 1, "box pairs reach at most one pair past the rows", N, es);
                    const long rl = r0 - 1, rr = r0 + N;
                    expect(rl >= 0 && rr < U * N, "u-trace rows inside the state", N, es);
                }
            }
        }
    }
}

// the order-8 fragment kernel's tile boxes and staged arrays (offsets from the stage start in
// issue order: tile, f^n tile, x faces, u faces, background tables, u-node speeds)
template <typename T>
void check_frag() {
    using G = vl::FragGeom<T>;
    const int es = (int)sizeof(T);
    expect(G::W <= 256 && G::WF <= 256 && G::COLS <= 256, "fragment boxes <= 256 elements wide", 8, es);
    expect((G::W * sizeof(T)) % 16 == 0 && (G::WF * sizeof(T)) % 16 == 0 && (G::COLS * sizeof(T)) % 16 == 0,
           "fragment box inner extents are 16-byte multiples", 8, es);
    expect(G::P * sizeof(T) == 16, "tile pad is one 16-byte unit", 8, es);
    expect(G::IN_B % 128 == 0 && G::FN_B % 128 == 0 && G::XF_B % 128 == 0 && G::UF_B % 128 == 0 &&
               G::BG_B % 128 == 0 && G::UX_B % 128 == 0 && G::STAGE_B % 128 == 0,
           "every fragment-kernel array starts on a 128-byte boundary", 8, es);
    expect((sizeof(T) * (size_t)G::COLS * 8) % 128 == 0, "second face side starts on a 128-byte boundary", 8, es);
    expect(G::smem_bytes() <= 227 * 1024, "fragment stage ring fits the shared memory of one CTA", 8, es);
}

template <int N>
void check_order() {
    check_tma<N, double>();
    check_tma<N, float>();
    check_pair<N>();
}

int main() {
    check_frag<double>();
    check_frag<float>();
    check_order<1>();
    check_order<2>();
    check_order<3>();
    check_order<4>();
    check_order<5>();
    check_order<6>();
    check_order<7>();
    check_order<8>();
    check_order<9>();
    check_order<10>();
    if (failures == 0) std::printf("ALL OK\n");
    return failures == 0 ? 0 : 1;
}
