// Halo-plan invariants under AddressSanitizer and UndefinedBehaviorSanitizer
// (built and run by tests/test_sanitizers.py, host code only).  For every
// rank of a range of decompositions and every level: each external column is a
// neighbour's row that this rank's stencil reaches, numbered as the plan says;
// every send list is the partner's receive list (same global ids, same order);
// halo rows and their external columns are in range and ascending.  Exits 0
// when everything holds, 1 with a message otherwise.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dist.hpp"

using namespace hpcg_b200;

static int fails = 0;
#define CHECK(c, ...)                         \
    do                                        \
    {                                         \
        if(!(c))                              \
        {                                     \
            if(fails++ < 10)                  \
            {                                 \
                std::fprintf(stderr, __VA_ARGS__); \
                std::fprintf(stderr, "\n");   \
            }                                 \
        }                                     \
    } while(0)

static long long gid_of(const DistGeom& g, int row)
{
    const int ix = row % g.nx, iy = (row / g.nx) % g.ny, iz = row / (g.nx * g.ny);
    return ((g.giz0 + iz) * g.gny + (g.giy0 + iy)) * g.gnx + (g.gix0 + ix);
}

static void check_decomposition(int size, int npx, int npy, int npz, int nx, int ny, int nz, int levels)
{
    std::vector<DistGeom> geo(size);
    for(int r = 0; r < size; ++r) geo[r] = make_geom(size, r, npx, npy, npz, nx, ny, nz);
    for(int l = 0; l < levels; ++l)
    {
        std::vector<HaloPlan> P(size);
        for(int r = 0; r < size; ++r) P[r] = plan_halo(geo[r]);
        for(int r = 0; r < size; ++r)
        {
            const DistGeom& g = geo[r];
            const HaloPlan& p = P[r];
            CHECK(p.m == g.nx * g.ny * g.nz, "rank %d level %d: m", r, l);
            CHECK((int)p.recv_gid.size() == p.next, "rank %d level %d: recv_gid size", r, l);
            for(size_t j = 0; j < p.nbr_rank.size(); ++j)
            {
                const int q = p.nbr_rank[j];
                CHECK(q >= 0 && q < size && q != r, "rank %d: neighbour %d", r, q);
                // ascending global ids per neighbour
                for(int e = p.recv_off[j] + 1; e < p.recv_off[j] + p.recv_len[j]; ++e)
                    CHECK(p.recv_gid[e - 1] < p.recv_gid[e], "rank %d: receive ids not ascending", r);
                // the partner's send list to r, as global ids, is this receive list
                const HaloPlan& o = P[q];
                size_t k = 0;
                while(k < o.nbr_rank.size() && o.nbr_rank[k] != r) ++k;
                CHECK(k < o.nbr_rank.size(), "rank %d: %d does not list it as neighbour", r, q);
                if(k == o.nbr_rank.size()) continue;
                CHECK(o.send_len[k] == p.recv_len[j], "rank %d <- %d: lengths %d %d", r, q, o.send_len[k],
                      p.recv_len[j]);
                const int n = o.send_len[k] < p.recv_len[j] ? o.send_len[k] : p.recv_len[j];
                for(int i = 0; i < n; ++i)
                {
                    const int row = o.send_rows[o.send_off[k] + i];
                    CHECK(row >= 0 && row < o.m, "rank %d: send row %d out of range", q, row);
                    CHECK(gid_of(geo[q], row) == p.recv_gid[p.recv_off[j] + i], "rank %d <- %d: entry %d", r, q, i);
                }
            }
            // halo rows ascending, their external columns ascending and in range
            CHECK((int)p.halo_ptr.size() == (int)p.halo_rows.size() + 1, "rank %d: halo_ptr", r);
            for(size_t h = 0; h < p.halo_rows.size(); ++h)
            {
                CHECK(p.halo_rows[h] >= 0 && p.halo_rows[h] < p.m, "rank %d: halo row", r);
                if(h) CHECK(p.halo_rows[h - 1] < p.halo_rows[h], "rank %d: halo rows not ascending", r);
                CHECK(p.halo_ptr[h + 1] - p.halo_ptr[h] <= p.halo_width, "rank %d: halo width", r);
                for(int c = p.halo_ptr[h]; c < p.halo_ptr[h + 1]; ++c)
                {
                    CHECK(p.halo_cols[c] >= p.m && p.halo_cols[c] < p.m + p.next, "rank %d: halo column", r);
                    if(c > p.halo_ptr[h]) CHECK(p.halo_cols[c - 1] < p.halo_cols[c], "rank %d: columns order", r);
                }
            }
        }
        for(int r = 0; r < size; ++r) geo[r] = coarsen(geo[r]);
    }
}

int main()
{
    for(int size = 1; size <= 12; ++size)
    {
        int px, py, pz;
        optimal_shape(size, px, py, pz);
        CHECK(px * py * pz == size, "shape of %d", size);
        check_decomposition(size, px, py, pz, 8, 8, 8, 3);
        check_decomposition(size, px, py, pz, 16, 8, 8, 4);
    }
    check_decomposition(4, 1, 2, 2, 24, 16, 8, 4);
    check_decomposition(6, 1, 2, 3, 8, 8, 8, 3);
    check_decomposition(8, 2, 2, 2, 4, 4, 4, 2);
    check_decomposition(27, 3, 3, 3, 4, 4, 4, 1);
    if(fails) std::fprintf(stderr, "%d halo-plan checks failed\n", fails);
    else std::printf("halo plans: all checks hold\n");
    return fails ? 1 : 0;
}
