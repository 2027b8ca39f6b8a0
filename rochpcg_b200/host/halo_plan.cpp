// Process grid and halo plan of the domain decomposition (host only, no
// device work: the C ABI exposes both without a GPU).
#include <algorithm>
#include <cmath>
#include <map>
#include <stdexcept>

#include "dist.hpp"

namespace hpcg_b200 {

namespace {

// Prime factors with multiplicity, ascending (src/ComputeOptimalShapeXYZ.cpp:
// 47-72: the trial divisors stop at sqrt of the original n, plus one; what is
// left above 1 -- or 1 itself when nothing divided -- is the last factor).
std::map<int, int> prime_factors(int n)
{
    std::map<int, int> f;
    const int limit = (int)std::sqrt((double)n) + 1;
    while(n > 1 && (n & 1) == 0)
    {
        ++f[2];
        n >>= 1;
    }
    for(int d = 3; d <= limit; d += 2)
        while(n % d == 0)
        {
            ++f[d];
            n /= d;
        }
    if(n > 1 || f.empty()) ++f[n];
    return f;
}

int ipow(int b, int e)
{
    int v = 1;
    while(e-- > 0) v *= b;
    return v;
}

// Every way to take a nonzero number of each prime (up to `avail`), in the
// order of a mixed-radix counter whose first digit is the smallest prime
// (src/MixedBaseCounter.cpp:37-60): f(counts) is called per combination.
template <typename F>
void each_subset(const std::vector<int>& avail, F&& f)
{
    std::vector<int> cur(avail.size(), 0);
    for(;;)
    {
        size_t i = 0;
        for(; i < cur.size(); ++i)
        {
            if(++cur[i] <= avail[i]) break;
            cur[i] = 0;
        }
        if(i == cur.size()) return;  // wrapped to zero: every combination seen
        f(cur);
    }
}

}  // namespace

void optimal_shape(int size, int& npx, int& npy, int& npz)
{
    if(size < 1) throw std::invalid_argument("optimal_shape: size < 1");
    const std::map<int, int> f = prime_factors(size);
    std::vector<int> primes, counts;
    for(const auto& kv : f)
    {
        primes.push_back(kv.first);
        counts.push_back(kv.second);
    }
    if(primes.size() == 1)
    {
        const int p = primes[0], c = counts[0];
        npz = ipow(p, c / 3);
        npy = ipow(p, c / 3 + (c % 3 >= 2 ? 1 : 0));
        npx = ipow(p, c / 3 + (c % 3 >= 1 ? 1 : 0));
        return;
    }
    if(primes.size() == 2 && counts[0] == 1 && counts[1] == 1)
    {
        npx = primes[0], npy = primes[1], npz = 1;
        return;
    }
    if(primes.size() == 2 && counts[0] + counts[1] == 3)
    {
        npx = primes[0], npy = primes[1];
        npz = counts[0] == 2 ? primes[0] : primes[1];
        return;
    }
    if(primes.size() == 3 && counts[0] == 1 && counts[1] == 1 && counts[2] == 1)
    {
        npx = primes[0], npy = primes[1], npz = primes[2];
        return;
    }
    // least surface x*y + y*z + x*z over the splits into three factors; the
    // first split (in counter order) of least surface wins
    auto product = [&](const std::vector<int>& c) {
        int v = 1;
        for(size_t i = 0; i < c.size(); ++i) v *= ipow(primes[i], c[i]);
        return v;
    };
    double best = 2.0 * size + 1.0;
    each_subset(counts, [&](const std::vector<int>& c1) {
        std::vector<int> rest(counts.size());
        for(size_t i = 0; i < counts.size(); ++i) rest[i] = counts[i] - c1[i];
        each_subset(rest, [&](const std::vector<int>& c2) {
            const int t1 = product(c1), t2 = product(c2), t3 = size / t1 / t2;
            const double area = t1 * (double)t2 + t2 * (double)t3 + t1 * (double)t3;
            if(area < best)
            {
                best = area;
                npx = t1, npy = t2, npz = t3;
            }
        });
    });
}

DistGeom make_geom(int size, int rank, int npx, int npy, int npz, int nx, int ny, int nz)
{
    if(npx < 1 || npy < 1 || npz < 1 || npx * npy * npz != size)
        throw std::invalid_argument("process grid does not match the rank count");
    if(rank < 0 || rank >= size) throw std::invalid_argument("rank out of range");
    DistGeom g;
    g.size = size, g.rank = rank;
    g.npx = npx, g.npy = npy, g.npz = npz;
    g.ipz = rank / (npx * npy);
    g.ipy = (rank - g.ipz * npx * npy) / npx;
    g.ipx = rank % npx;
    g.nx = nx, g.ny = ny, g.nz = nz;
    g.gnx = (long long)npx * nx, g.gny = (long long)npy * ny, g.gnz = (long long)npz * nz;
    g.gix0 = (long long)g.ipx * nx, g.giy0 = (long long)g.ipy * ny, g.giz0 = (long long)g.ipz * nz;
    return g;
}

DistGeom coarsen(const DistGeom& g)
{
    return make_geom(g.size, g.rank, g.npx, g.npy, g.npz, g.nx / 2, g.ny / 2, g.nz / 2);
}

HaloPlan plan_halo(const DistGeom& g)
{
    HaloPlan P;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    P.m = nx * ny * nz;
    // per slot: the (global id) columns received, and the rows sent
    std::vector<std::vector<long long>> recv(27);
    std::vector<std::vector<int>> send(27);
    struct Entry
    {
        int slot;
        long long gid;
    };
    std::vector<Entry> entries;  // external entries of the halo rows, row by row
    std::vector<int> entry_ptr{0};

    auto visit = [&](int ix, int iy, int iz) {
        const long long gx = g.gix0 + ix, gy = g.giy0 + iy, gz = g.giz0 + iz;
        const int row = (iz * ny + iy) * nx + ix;
        unsigned int sent = 0;
        const size_t before = entries.size();
        for(int dz = -1; dz <= 1; ++dz)
            for(int dy = -1; dy <= 1; ++dy)
                for(int dx = -1; dx <= 1; ++dx)
                {
                    const long long cx = gx + dx, cy = gy + dy, cz = gz + dz;
                    if(cx < 0 || cy < 0 || cz < 0 || cx >= g.gnx || cy >= g.gny || cz >= g.gnz) continue;
                    const int ox = ix + dx < 0 ? -1 : (ix + dx >= nx ? 1 : 0);
                    const int oy = iy + dy < 0 ? -1 : (iy + dy >= ny ? 1 : 0);
                    const int oz = iz + dz < 0 ? -1 : (iz + dz >= nz ? 1 : 0);
                    if(!ox && !oy && !oz) continue;  // a local column
                    const int slot = (oz + 1) * 9 + (oy + 1) * 3 + (ox + 1);
                    const long long gid = (cz * g.gny + cy) * g.gnx + cx;
                    recv[slot].push_back(gid);
                    entries.push_back({slot, gid});
                    if(!(sent & (1u << slot)))
                    {
                        sent |= 1u << slot;
                        send[slot].push_back(row);  // rows are visited in ascending order
                    }
                }
        if(entries.size() != before)
        {
            P.halo_rows.push_back(row);
            entry_ptr.push_back((int)entries.size());
        }
    };
    // only surface rows can have external columns
    for(int iz = 0; iz < nz; ++iz)
        for(int iy = 0; iy < ny; ++iy)
        {
            if(iz == 0 || iz == nz - 1 || iy == 0 || iy == ny - 1)
                for(int ix = 0; ix < nx; ++ix) visit(ix, iy, iz);
            else
            {
                visit(0, iy, iz);
                if(nx > 1) visit(nx - 1, iy, iz);
            }
        }

    // neighbours in slot order; external ids numbered neighbour by neighbour
    std::vector<int> base(27, -1);
    int next = 0, sent_total = 0;
    for(int s = 0; s < 27; ++s)
    {
        auto& r = recv[s];
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
        if(r.empty()) continue;
        if(send[s].empty()) throw std::logic_error("halo plan: a neighbour receives without sending");
        const int dz = s / 9 - 1, dy = (s / 3) % 3 - 1, dx = s % 3 - 1;
        P.nbr_slot.push_back(s);
        P.nbr_rank.push_back(g.rank_at(g.ipx + dx, g.ipy + dy, g.ipz + dz));
        P.recv_off.push_back(next);
        P.recv_len.push_back((int)r.size());
        P.send_off.push_back(sent_total);
        P.send_len.push_back((int)send[s].size());
        base[s] = next;
        next += (int)r.size();
        sent_total += (int)send[s].size();
        P.recv_gid.insert(P.recv_gid.end(), r.begin(), r.end());
        P.send_rows.insert(P.send_rows.end(), send[s].begin(), send[s].end());
    }
    P.next = next;

    // the external columns of each halo row, ascending
    P.halo_ptr.push_back(0);
    for(size_t h = 0; h < P.halo_rows.size(); ++h)
    {
        const int b = entry_ptr[h], e = entry_ptr[h + 1];
        std::vector<int> cols;
        for(int i = b; i < e; ++i)
        {
            const auto& r = recv[entries[i].slot];
            const int k = (int)(std::lower_bound(r.begin(), r.end(), entries[i].gid) - r.begin());
            cols.push_back(P.m + base[entries[i].slot] + k);
        }
        std::sort(cols.begin(), cols.end());
        P.halo_cols.insert(P.halo_cols.end(), cols.begin(), cols.end());
        P.halo_ptr.push_back((int)P.halo_cols.size());
        P.halo_width = std::max(P.halo_width, (int)cols.size());
    }
    return P;
}

}  // namespace hpcg_b200
