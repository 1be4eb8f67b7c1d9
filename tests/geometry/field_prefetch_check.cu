// Host check (no GPU) of the cluster field solve's table prefetch (vlasov_field.cuh): for every
// order n <= 10, every element count with nx n within the solver's capacity, a range of mode
// counts up to the capacity and every cluster rank, the entries each CTA copies and reads stay
// inside its shared-memory regions and inside the global tables, the regions add up to the
// launch's dynamic shared memory, and that fits the per-CTA limit beside the kernel's static
// shared memory.  Mirrors the index arithmetic of field_cluster_body.
#include <cstdio>

#include "vlasov_field.cuh"

static long failures = 0;

static void expect(bool ok, const char *what, int nx, int n, int M, int rank) {
    if (!ok) {
        if (failures < 20) std::printf("FAIL %s: nx=%d n=%d M=%d rank=%d\n", what, nx, n, M, rank);
        ++failures;
    }
}

// kernel static shared memory upper bound (s_rhs, s_E, s_P, s_fold, reductions): 19904 bytes
// reported by ptxas for field_solve_kernel; the check keeps 1 KB of margin
constexpr size_t kStaticMax = 21 * 1024;
constexpr size_t kSmemPerCta = 227 * 1024;

static void check(int nx, int n, int M) {
    using namespace vl;
    const int nn = nx * n;
    const int Mc = field_fwd_cols(M);
    const int Nc = (nn + FC - 1) / FC;
    const size_t pre = field_prefetch_bytes(nx, n, M);
    for (int phi = 0; phi < 2; ++phi) {
        const size_t base = field_solve_smem_for(n, M, phi != 0);
        const bool prefetch = base + pre <= FIELD_DYN_SMEM_MAX;
        expect(base <= field_solve_smem(n, M), "base within the attribute", nx, n, M, -1);
        if (!prefetch) continue;
        // region offsets in double2 entries, as in field_cluster_body
        const size_t oPF = (size_t)(phi ? 2 : 1) * n * M;
        const size_t oPI = oPF + (size_t)nx * Mc;
        const size_t oEL = oPI + (size_t)field_inv_rows(nx, n) * M;
        const size_t oQN = oEL + (size_t)n * Mc;
        const size_t end = oQN + (size_t)n * M;
        expect(end * sizeof(double2) == base + pre, "regions add up to the dynamic size", nx, n, M, -1);
        for (int rank = 0; rank < FC; ++rank) {
            const int m0 = rank * Mc;
            const int p0 = rank * Nc;
            const int e_lo = p0 < nn ? p0 / n : 0;
            const int e_hi = p0 < nn ? ((p0 + Nc < nn ? p0 + Nc : nn) - 1) / n : -1;
            const int rows = e_hi - e_lo + 1;
            expect(rows >= 0 && rows <= field_inv_rows(nx, n), "inverse rows fit their region", nx, n, M, rank);
            expect(e_hi < nx, "inverse rows inside the phase table", nx, n, M, rank);
            // forward copies: entry q = e Mc + ml of phase[e][m0 + ml] for m0 + ml < M
            if (Mc > 0) {
                const long last_f = (long)(nx - 1) * M + (m0 + Mc - 1 < M ? m0 + Mc - 1 : M - 1);
                expect(m0 >= M || last_f < (long)nx * M, "forward copy inside the phase table", nx, n, M, rank);
                const long last_l = (long)(n - 1) * M + (m0 + Mc - 1 < M ? m0 + Mc - 1 : M - 1);
                expect(m0 >= M || last_l < (long)n * M, "ell copy inside the ell table", nx, n, M, rank);
            }
            // inverse reads: node p in [p0, min(p0 + Nc, nn)) reads row e - e_lo of its element
            for (int p = p0; p < p0 + Nc && p < nn; ++p) {
                const int e = p / n;
                expect(e >= e_lo && e <= e_hi, "node's element among the copied rows", nx, n, M, rank);
            }
        }
    }
}

int main() {
    using namespace vl;
    static_assert(FIELD_DYN_SMEM_MAX + kStaticMax <= kSmemPerCta, "dynamic budget beside static shared memory");
    static_assert(2 * NMAX * FIELD_MAX_MODES * sizeof(double2) + kStaticMax <= kSmemPerCta,
                  "the solve without prefetch at the capacity");
    const int modes[] = {1, 2, 3, 7, 8, 9, 15, 16, 17, 63, 64, 65, 159, 160, 161, 255, 287, 319, 320, FIELD_MAX_MODES};
    long cases = 0;
    for (int n = 1; n <= NMAX; ++n)
        for (int nx = 1; nx * n <= FIELD_MAX_NODES; ++nx)
            for (int M : modes) {
                check(nx, n, M);
                ++cases;
            }
    if (failures) {
        std::printf("%ld failures in %ld cases\n", failures, cases);
        return 1;
    }
    std::printf("ALL OK (%ld cases)\n", cases);
    return 0;
}
