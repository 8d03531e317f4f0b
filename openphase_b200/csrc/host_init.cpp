// Host-side initial states and raw-file IO for the opgpu C ABI (no GPU needed).
//
//  * opgpu_uniform                  counter-based uniform variate (opgpu_rng.h)
//  * opgpu_voronoi_owner_host       seeded periodic Voronoi owner map
//  * opgpu_spread_boundaries_host   grain-boundary spreading into per-voxel lists
//  * raw PhaseField file read/write helpers used by opgpu_read_raw / opgpu_write_raw
//
// The Voronoi search prunes seeds per block of voxels: for each 8^3 block the largest possible
// distance to the nearest seed bounds the candidate set, then every voxel scans only the
// candidates.  The result is exactly the brute-force argmin (ties to the lowest grain index).
#include "opgpu.h"
#include "opgpu_rng.h"
#include "opgpu_host.h"

#include <omp.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <vector>

extern "C" double opgpu_uniform(uint64_t seed, uint64_t stream, uint64_t a, uint64_t b)
{
    return opgpu::uniform01(seed, stream, a, b);
}

namespace {

inline int pdist(int a, int b, int n)
{
    int d = a > b ? a - b : b - a;
    return d < n - d ? d : n - d;
}

void set_threads(int threads)
{
    if (threads > 0) omp_set_num_threads(threads);
}

}  // namespace

extern "C" uint32_t opgpu_voronoi_owner_host(int32_t nx, int32_t ny, int32_t nz, int32_t ngrains,
                                             uint64_t seed, int32_t threads, int32_t* owner)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || ngrains <= 0 || !owner) return OPGPU_E_INVALID;
    set_threads(threads);
    const int G = ngrains;
    std::vector<int> sx(G), sy(G), sz(G);
    const int dims[3] = {nx, ny, nz};
    for (int g = 0; g < G; g++)
    {
        int c[3];
        for (int a = 0; a < 3; a++)
        {
            int v = (int)(opgpu::uniform01(seed, opgpu::kStreamPosition, (uint64_t)g, (uint64_t)a) * dims[a]);
            c[a] = v < dims[a] ? v : dims[a] - 1;
        }
        sx[g] = c[0]; sy[g] = c[1]; sz[g] = c[2];
    }
    const int B = 8;
    const int bx = (nx + B - 1) / B, by = (ny + B - 1) / B, bz = (nz + B - 1) / B;
    const long nblocks = (long)bx * by * bz;
    #pragma omp parallel
    {
        std::vector<int> cand;
        std::vector<long> dmin(G);
        #pragma omp for schedule(dynamic, 4)
        for (long blk = 0; blk < nblocks; blk++)
        {
            const int ib = (int)(blk / ((long)by * bz));
            const int jb = (int)((blk / bz) % by);
            const int kb = (int)(blk % bz);
            const int lo[3] = {ib * B, jb * B, kb * B};
            const int hi[3] = {std::min(lo[0] + B, nx), std::min(lo[1] + B, ny), std::min(lo[2] + B, nz)};
            long best_max = LONG_MAX;
            for (int g = 0; g < G; g++)
            {
                const int s[3] = {sx[g], sy[g], sz[g]};
                long mn = 0, mx = 0;
                for (int a = 0; a < 3; a++)
                {
                    int amin = INT_MAX, amax = 0;
                    for (int p = lo[a]; p < hi[a]; p++)
                    {
                        const int d = pdist(p, s[a], dims[a]);
                        amin = std::min(amin, d);
                        amax = std::max(amax, d);
                    }
                    mn += (long)amin * amin;
                    mx += (long)amax * amax;
                }
                dmin[g] = mn;
                best_max = std::min(best_max, mx);
            }
            cand.clear();
            for (int g = 0; g < G; g++) if (dmin[g] <= best_max) cand.push_back(g);
            for (int i = lo[0]; i < hi[0]; i++)
            for (int j = lo[1]; j < hi[1]; j++)
            for (int k = lo[2]; k < hi[2]; k++)
            {
                long best = LONG_MAX;
                int bg = -1;
                for (int g : cand)   // ascending g: strict < keeps the lowest index on ties
                {
                    const long dx = pdist(i, sx[g], nx), dy = pdist(j, sy[g], ny), dz = pdist(k, sz[g], nz);
                    const long d = dx * dx + dy * dy + dz * dz;
                    if (d < best) { best = d; bg = g; }
                }
                owner[((long)i * ny + j) * nz + k] = bg;
            }
        }
    }
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_spread_boundaries_host(int32_t nx, int32_t ny, int32_t nz, const int32_t* owner,
                                                 int32_t threads, int32_t* counts, int32_t* idx,
                                                 int64_t* total)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || !owner || !counts) return OPGPU_E_INVALID;
    set_threads(threads);
    const long n = (long)nx * ny * nz;
    auto lists = [&](long v, int32_t* out) -> int {
        const int i = (int)(v / ((long)ny * nz)), j = (int)((v / nz) % ny), k = (int)(v % nz);
        int m = 0;
        int32_t loc[27];
        loc[m++] = owner[v];
        for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++)
        for (int dk = -1; dk <= 1; dk++)
        {
            if (!di && !dj && !dk) continue;
            const long u = (((long)((i + di + nx) % nx)) * ny + (j + dj + ny) % ny) * nz + (k + dk + nz) % nz;
            const int32_t g = owner[u];
            bool seen = false;
            for (int q = 0; q < m; q++) if (loc[q] == g) { seen = true; break; }
            if (!seen) loc[m++] = g;
        }
        if (out) std::memcpy(out, loc, m * sizeof(int32_t));
        return m;
    };
    if (!idx)
    {
        int64_t t = 0;
        #pragma omp parallel for reduction(+:t) schedule(static)
        for (long v = 0; v < n; v++) { counts[v] = lists(v, nullptr); t += counts[v]; }
        if (total) *total = t;
        return OPGPU_OK;
    }
    // second pass: offsets from the counts computed by the first pass
    std::vector<int64_t> off(n + 1, 0);
    for (long v = 0; v < n; v++) off[v + 1] = off[v] + counts[v];
    #pragma omp parallel for schedule(static)
    for (long v = 0; v < n; v++) lists(v, idx + off[v]);
    if (total) *total = off[n];
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_pair_table_host(int32_t ngrains, uint64_t seed, uint64_t stream, double lo,
                                          double span, double* out)
{
    if (ngrains <= 0 || !out) return OPGPU_E_INVALID;
    const long G = ngrains;
    #pragma omp parallel for schedule(dynamic, 16)
    for (long a = 0; a < G; a++)
    {
        out[a * G + a] = lo;
        for (long b = a + 1; b < G; b++)
        {
            const double v = lo + span * opgpu::uniform01(seed, stream, (uint64_t)a, (uint64_t)b);
            out[a * G + b] = v;
            out[b * G + a] = v;
        }
    }
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_grain_values_host(int32_t ngrains, uint64_t seed, uint64_t stream, double scale,
                                            double* out)
{
    if (ngrains <= 0 || !out) return OPGPU_E_INVALID;
    for (int g = 0; g < ngrains; g++) out[g] = scale * opgpu::uniform01(seed, stream, (uint64_t)g, 0);
    return OPGPU_OK;
}

namespace opgpu {

// Raw PhaseField format (src/PhaseField.cpp:2340-2388, NodePF::write NodePF.h:765-775):
// int32 Nx, Ny, Nz; then per voxel size_t n and n x (size_t index, double value).
bool raw_read(const char* path, int nx, int ny, int nz, std::vector<int32_t>& counts,
              std::vector<int32_t>& idx, std::vector<double>& val, std::string& err)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) { err = std::string("cannot open ") + path; return false; }
    int32_t hdr[3];
    if (std::fread(hdr, sizeof(int32_t), 3, f) != 3 || hdr[0] != nx || hdr[1] != ny || hdr[2] != nz)
    {
        std::fclose(f);
        err = "raw file dimensions do not match the grid";
        return false;
    }
    const long n = (long)nx * ny * nz;
    counts.assign(n, 0);
    idx.clear(); val.clear();
    idx.reserve(n * 3); val.reserve(n * 3);
    for (long v = 0; v < n; v++)
    {
        uint64_t c = 0;
        if (std::fread(&c, sizeof(uint64_t), 1, f) != 1 || c > 4096)
        {
            std::fclose(f);
            err = "truncated or corrupt raw file";
            return false;
        }
        counts[v] = (int32_t)c;
        for (uint64_t q = 0; q < c; q++)
        {
            uint64_t g; double x;
            if (std::fread(&g, sizeof(uint64_t), 1, f) != 1 || std::fread(&x, sizeof(double), 1, f) != 1
                || g > (uint64_t)INT32_MAX)
            {
                std::fclose(f);
                err = "truncated or corrupt raw file";
                return false;
            }
            idx.push_back((int32_t)g);
            val.push_back(x);
        }
    }
    std::fclose(f);
    return true;
}

bool raw_write(const char* path, int nx, int ny, int nz, const int32_t* counts, const int32_t* idx,
               const double* val, std::string& err)
{
    FILE* f = std::fopen(path, "wb");
    if (!f) { err = std::string("cannot open ") + path; return false; }
    const int32_t hdr[3] = {nx, ny, nz};
    bool ok = std::fwrite(hdr, sizeof(int32_t), 3, f) == 3;
    const long n = (long)nx * ny * nz;
    long off = 0;
    std::vector<unsigned char> buf;
    for (long v = 0; v < n && ok; v++)
    {
        const uint64_t c = (uint64_t)counts[v];
        buf.resize(8 + c * 16);
        std::memcpy(buf.data(), &c, 8);
        for (uint64_t q = 0; q < c; q++)
        {
            const uint64_t g = (uint64_t)idx[off + q];
            std::memcpy(buf.data() + 8 + q * 16, &g, 8);
            std::memcpy(buf.data() + 16 + q * 16, &val[off + q], 8);
        }
        off += (long)c;
        ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) err = std::string("write failed: ") + path;
    return ok;
}

}  // namespace opgpu
