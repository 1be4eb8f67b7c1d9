// Host-side check of the shared-memory and tensor-copy geometry of the fragment kernel (n = 8)
// and of the generic stage kernel's TMA form, for every compiled order and both precisions: box
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
