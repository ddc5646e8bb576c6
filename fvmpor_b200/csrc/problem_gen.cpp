// Synthetic Richards problems: jittered-grid Delaunay triangulations (2D),
// Kuhn 6-tet splits of jittered hex grids (3D), lognormal conductivity
// fields by circulant-embedding FFT, soil zones, boundary tags and the
// hydrostatic initial state.
//
// The reference builds its meshes offline with gmsh and decomp
// (meshing/genMesh.sh, decomp/split.c:459-500) and reads them in
// src/fvm/mesh.cpp:82-366.  This file produces the same mesh description
// (node coordinates, element connectivity with zone tags, boundary faces
// with boundary tags, per-node Dirichlet tags) for the seeded benchmark
// problems directly.  Nodes are numbered tile by tile so that contiguous
// node ranges are spatially compact; the block preconditioner and the
// gather kernels rely on that locality.
#include "common.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <numeric>
#include <vector>

namespace fvmb {

// ---------------------------------------------------------------- RNG
Rng::Rng(uint64_t seed) : s(seed ^ 0x9E3779B97F4A7C15ull) { next(); next(); }
uint64_t Rng::next() {
    // splitmix64
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double Rng::uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
double Rng::normal() {
    if (has_spare) { has_spare = false; return spare; }
    double u1, u2;
    do { u1 = uniform(); } while (u1 <= 0.0);
    u2 = uniform();
    double r = std::sqrt(-2.0 * std::log(u1));
    spare = r * std::sin(2.0 * M_PI * u2);
    has_spare = true;
    return r * std::cos(2.0 * M_PI * u2);
}

// ---------------------------------------------------------------- FFT
using cd = std::complex<double>;

static void fft_inplace(cd* a, int n) {
    // iterative radix-2 Cooley-Tukey, forward transform (e^{-i...})
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
        double ang = -2.0 * M_PI / len;
        cd wl(std::cos(ang), std::sin(ang));
        for (int i = 0; i < n; i += len) {
            cd w(1.0, 0.0);
            for (int k = 0; k < len / 2; ++k) {
                cd u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
                w *= wl;
            }
        }
    }
}

// forward DFT over a dense n0 x n1 x n2 array (index i0 + n0*(i1 + n1*i2))
static void fft3(std::vector<cd>& a, int n0, int n1, int n2) {
    std::vector<cd> line(std::max(n0, std::max(n1, n2)));
    for (int i2 = 0; i2 < n2; ++i2)
        for (int i1 = 0; i1 < n1; ++i1) fft_inplace(&a[(size_t)n0 * (i1 + (size_t)n1 * i2)], n0);
    if (n1 > 1)
        for (int i2 = 0; i2 < n2; ++i2)
            for (int i0 = 0; i0 < n0; ++i0) {
                for (int i1 = 0; i1 < n1; ++i1) line[i1] = a[i0 + (size_t)n0 * (i1 + (size_t)n1 * i2)];
                fft_inplace(line.data(), n1);
                for (int i1 = 0; i1 < n1; ++i1) a[i0 + (size_t)n0 * (i1 + (size_t)n1 * i2)] = line[i1];
            }
    if (n2 > 1)
        for (int i1 = 0; i1 < n1; ++i1)
            for (int i0 = 0; i0 < n0; ++i0) {
                for (int i2 = 0; i2 < n2; ++i2) line[i2] = a[i0 + (size_t)n0 * (i1 + (size_t)n1 * i2)];
                fft_inplace(line.data(), n2);
                for (int i2 = 0; i2 < n2; ++i2) a[i0 + (size_t)n0 * (i1 + (size_t)n1 * i2)] = line[i2];
            }
}

static int pow2_at_least(int n) { int p = 1; while (p < n) p <<= 1; return p; }

// Zero-mean stationary Gaussian field with exponential covariance
//   C(d) = var * exp(-sqrt((dx/Lx)^2 + (dy/Ly)^2 + (dz/Lz)^2))
// sampled at the centres of an nx*ny*nz cell grid of spacing (hx,hy,hz),
// by circulant embedding (Dietrich & Newsam 1997): embed the covariance in
// a periodic grid padded by about three correlation lengths, take its DFT
// (the circulant eigenvalues, negatives clipped to zero), colour complex
// white noise with their square roots and transform back; the real part
// has covariance C.
std::vector<double> gaussian_field(int nx, int ny, int nz, double hx, double hy, double hz,
                                   double var, double Lx, double Ly, double Lz, uint64_t seed) {
    std::vector<double> out((size_t)nx * ny * nz, 0.0);
    if (var <= 0.0) return out;
    int m0 = pow2_at_least(nx + (int)std::ceil(3.0 * Lx / hx));
    int m1 = ny > 1 ? pow2_at_least(ny + (int)std::ceil(3.0 * Ly / hy)) : 1;
    int m2 = nz > 1 ? pow2_at_least(nz + (int)std::ceil(3.0 * Lz / hz)) : 1;
    size_t M = (size_t)m0 * m1 * m2;
    std::vector<cd> lam(M);
    for (int i2 = 0; i2 < m2; ++i2)
        for (int i1 = 0; i1 < m1; ++i1)
            for (int i0 = 0; i0 < m0; ++i0) {
                double a = std::min(i0, m0 - i0) * hx / Lx;
                double b = m1 > 1 ? std::min(i1, m1 - i1) * hy / Ly : 0.0;
                double c = m2 > 1 ? std::min(i2, m2 - i2) * hz / Lz : 0.0;
                lam[i0 + (size_t)m0 * (i1 + (size_t)m1 * i2)] = cd(var * std::exp(-std::sqrt(a * a + b * b + c * c)), 0.0);
            }
    fft3(lam, m0, m1, m2);
    Rng rng(seed);
    std::vector<cd> z(M);
    for (size_t i = 0; i < M; ++i) {
        double l = std::max(lam[i].real(), 0.0);
        double s = std::sqrt(l / (double)M);
        double xr = rng.normal(), xi = rng.normal();
        z[i] = cd(s * xr, s * xi);
    }
    fft3(z, m0, m1, m2);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                out[i + (size_t)nx * (j + (size_t)ny * k)] = z[i + (size_t)m0 * (j + (size_t)m1 * k)].real();
    return out;
}

// ---------------------------------------------------------------- ordering
// Tile-major numbering of an nx*ny (x nz) node grid: tiles of tx*ty columns
// in row-major tile order; inside a tile columns row-major, z fastest.
static std::vector<int> tiled_order(int nx, int ny, int nz, int tx, int ty) {
    std::vector<int> perm((size_t)nx * ny * nz);
    int ntx = (nx + tx - 1) / tx, nty = (ny + ty - 1) / ty;
    int next = 0;
    for (int TJ = 0; TJ < nty; ++TJ)
        for (int TI = 0; TI < ntx; ++TI)
            for (int j = TJ * ty; j < std::min(ny, (TJ + 1) * ty); ++j)
                for (int i = TI * tx; i < std::min(nx, (TI + 1) * tx); ++i)
                    for (int k = 0; k < nz; ++k) perm[i + (size_t)nx * (j + (size_t)ny * k)] = next++;
    return perm;
}

static void* xmalloc(size_t n) {
    void* p = std::malloc(n ? n : 1);
    if (!p) throw Error("out of host memory");
    return p;
}
template <class T> static T* copy_out(const std::vector<T>& v) {
    T* p = (T*)xmalloc(v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

static void finish_problem(fvm_problem* out, int dim, const std::vector<double>& coords,
                           const std::vector<int>& en, const std::vector<int>& ez,
                           const std::vector<double>& eK, const std::vector<int>& bn,
                           const std::vector<int>& be, const std::vector<int>& bt,
                           const std::vector<int>& nt, const std::vector<fvm_zone>& zones,
                           const std::vector<fvm_bc>& bcs, int g0, int g1, int g2) {
    std::memset(out, 0, sizeof(*out));
    out->coords = copy_out(coords);
    out->elem_nodes = copy_out(en);
    out->elem_zone = copy_out(ez);
    out->elem_K = eK.empty() ? nullptr : copy_out(eK);
    out->bface_nodes = copy_out(bn);
    out->bface_elem = copy_out(be);
    out->bface_tag = copy_out(bt);
    out->node_tag = copy_out(nt);
    out->zones = copy_out(zones);
    out->bcs = copy_out(bcs);
    out->grid_dims = (int*)xmalloc(3 * sizeof(int));
    out->grid_dims[0] = g0; out->grid_dims[1] = g1; out->grid_dims[2] = g2;
    fvm_mesh& m = out->mesh;
    m.dim = dim;
    m.n_nodes = (int)(coords.size() / 3);
    m.n_elements = (int)(ez.size());
    m.n_bfaces = (int)bt.size();
    m.coords = out->coords; m.elem_nodes = out->elem_nodes; m.elem_zone = out->elem_zone;
    m.elem_K = out->elem_K; m.bface_nodes = out->bface_nodes; m.bface_elem = out->bface_elem;
    m.bface_tag = out->bface_tag; m.node_tag = out->node_tag;
    out->phys.n_zones = (int)zones.size();
    out->phys.zones = out->zones;
    out->phys.n_bcs = (int)bcs.size();
    out->phys.bcs = out->bcs;
    out->phys.rho0 = 1000.0;
}

// incircle determinant: > 0 when d lies inside the circle through the
// counter-clockwise triangle (a, b, c)
static double incircle(const double* a, const double* b, const double* c, const double* d) {
    double adx = a[0] - d[0], ady = a[1] - d[1];
    double bdx = b[0] - d[0], bdy = b[1] - d[1];
    double cdx = c[0] - d[0], cdy = c[1] - d[1];
    double ad = adx * adx + ady * ady, bd = bdx * bdx + bdy * bdy, cdd = cdx * cdx + cdy * cdy;
    return adx * (bdy * cdd - bd * cdy) - ady * (bdx * cdd - bd * cdx) + ad * (bdx * cdy - bdy * cdx);
}

static double orient2(const double* a, const double* b, const double* c) {
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]);
}

// Delaunay triangulation of a jittered nx*ny node grid.  With jitter below
// a quarter of the spacing, every Delaunay triangle lies inside one grid
// cell (grid edges keep a 90-degree margin in the opposite-angle test), so
// the triangulation is each cell split along its locally Delaunay diagonal.
static void build_2d(int nx, int ny, double Lx, double Ly, double jitter, uint64_t seed,
                     double x0, double y0, int tile, std::vector<double>& coords,
                     std::vector<int>& en, std::vector<int>& perm) {
    double hx = Lx / (nx - 1), hy = Ly / (ny - 1);
    Rng rng(seed);
    std::vector<double> xy((size_t)2 * nx * ny);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            double dx = (2.0 * rng.uniform() - 1.0) * jitter * hx;
            double dy = (2.0 * rng.uniform() - 1.0) * jitter * hy;
            if (i == 0 || i == nx - 1) dx = 0.0;
            if (j == 0 || j == ny - 1) dy = 0.0;
            xy[2 * (i + (size_t)nx * j)] = x0 + i * hx + dx;
            xy[2 * (i + (size_t)nx * j) + 1] = y0 + j * hy + dy;
        }
    perm = tiled_order(nx, ny, 1, tile, tile);
    size_t base = coords.size() / 3;
    coords.resize(coords.size() + (size_t)3 * nx * ny);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            size_t g = i + (size_t)nx * j, p = base + perm[g];
            coords[3 * p] = xy[2 * g];
            coords[3 * p + 1] = xy[2 * g + 1];
            coords[3 * p + 2] = 0.0;
        }
    // cells in tile-major order
    std::vector<int> corder = tiled_order(nx - 1, ny - 1, 1, tile, tile);
    std::vector<int> cells((size_t)(nx - 1) * (ny - 1));
    for (size_t c = 0; c < cells.size(); ++c) cells[corder[c]] = (int)c;
    for (int c : cells) {
        int i = c % (nx - 1), j = c / (nx - 1);
        int ga = i + nx * j, gb = ga + 1, gc = ga + 1 + nx, gd = ga + nx;
        const double *a = &xy[2 * ga], *b = &xy[2 * gb], *cc = &xy[2 * gc], *d = &xy[2 * gd];
        int tri[2][3];
        if (incircle(a, b, cc, d) <= 0.0) {
            int t0[3] = {ga, gb, gc}, t1[3] = {ga, gc, gd};
            std::memcpy(tri[0], t0, sizeof t0); std::memcpy(tri[1], t1, sizeof t1);
        } else {
            int t0[3] = {ga, gb, gd}, t1[3] = {gb, gc, gd};
            std::memcpy(tri[0], t0, sizeof t0); std::memcpy(tri[1], t1, sizeof t1);
        }
        for (auto& t : tri) {
            if (orient2(&xy[2 * t[0]], &xy[2 * t[1]], &xy[2 * t[2]]) <= 0.0)
                throw Error("jitter too large: degenerate triangle");
            for (int k = 0; k < 3; ++k) en.push_back((int)base + perm[t[k]]);
        }
    }
}

} // namespace fvmb

using namespace fvmb;

extern "C" int fvm_problem_richards2d(int nx, int ny, double Lx, double Ly, double jitter,
                                      uint64_t seed, double ln_var, double corr_len,
                                      fvm_problem* out) {
    try {
        if (nx < 2 || ny < 2 || !out || jitter < 0.0 || jitter >= 0.25)
            throw Error("fvm_problem_richards2d: bad arguments");
        std::vector<double> coords;
        std::vector<int> en, perm;
        build_2d(nx, ny, Lx, Ly, jitter, seed, 0.0, 0.0, 16, coords, en, perm);
        int N = nx * ny, T = (int)en.size() / 3;
        // zones split at mid-height: lower layer 0, upper layer 1
        std::vector<int> ez(T);
        for (int e = 0; e < T; ++e) {
            double yc = (coords[3 * en[3 * e] + 1] + coords[3 * en[3 * e + 1] + 1] + coords[3 * en[3 * e + 2] + 1]) / 3.0;
            ez[e] = yc < 0.5 * Ly ? 0 : 1;
        }
        std::vector<fvm_zone> zones(2);
        zones[0] = fvm_zone{1e-5, 1e-5, 1e-5, 0.40, 1.0, 2.0, 0.05 / 0.40};
        zones[1] = fvm_zone{1e-6, 1e-6, 1e-6, 0.45, 3.0, 1.6, 0.10 / 0.45};
        std::vector<double> eK;
        if (ln_var > 0.0) {
            int cx = nx - 1, cy = ny - 1;
            std::vector<double> f = gaussian_field(cx, cy, 1, Lx / cx, Ly / cy, 1.0, ln_var,
                                                   corr_len, corr_len, 1.0, seed ^ 0xA5A5A5A5ull);
            eK.resize(T);
            // element e belongs to cell: elements are emitted two per cell in
            // tile-major cell order; recover the cell from the centroid
            double hx = Lx / cx, hy = Ly / cy;
            for (int e = 0; e < T; ++e) {
                double xc = 0, yc = 0;
                for (int k = 0; k < 3; ++k) { xc += coords[3 * en[3 * e + k]]; yc += coords[3 * en[3 * e + k] + 1]; }
                xc /= 3; yc /= 3;
                int ci = std::min(cx - 1, std::max(0, (int)(xc / hx)));
                int cj = std::min(cy - 1, std::max(0, (int)(yc / hy)));
                eK[e] = zones[ez[e]].Kxx * std::exp(f[ci + (size_t)cx * cj]);
            }
        }
        // boundary tags: 1 = no flow, 2 = Dirichlet h = 0 on the top strip
        // 4 <= x <= 6 (scaled with the domain width: 0.4 Lx .. 0.6 Lx)
        std::vector<int> nt(N, 0);
        auto gid = [&](int i, int j) { return perm[i + (size_t)nx * j]; };
        for (int i = 0; i < nx; ++i) {
            int n = gid(i, ny - 1);
            double x = coords[3 * n];
            if (x >= 0.4 * Lx - 1e-12 && x <= 0.6 * Lx + 1e-12) nt[n] = 2;
        }
        // boundary segments with their owning triangle
        std::vector<int> bn, be, bt;
        {
            // map sorted node pair -> element
            std::vector<std::vector<std::pair<int, int>>> adj(N);
            for (int e = 0; e < T; ++e)
                for (int k = 0; k < 3; ++k) {
                    int a = en[3 * e + k], b = en[3 * e + (k + 1) % 3];
                    adj[std::min(a, b)].push_back({std::max(a, b), e});
                }
            auto owner = [&](int a, int b) {
                for (auto& pr : adj[std::min(a, b)]) if (pr.first == std::max(a, b)) return pr.second;
                throw Error("boundary segment without element");
            };
            auto add = [&](int a, int b, int tag) {
                int e = owner(a, b);
                bn.push_back(a); bn.push_back(b); be.push_back(e); bt.push_back(tag);
            };
            for (int i = 0; i + 1 < nx; ++i) add(gid(i, 0), gid(i + 1, 0), 1);                 // bottom
            for (int j = 0; j + 1 < ny; ++j) add(gid(nx - 1, j), gid(nx - 1, j + 1), 1);       // right
            for (int i = nx - 1; i > 0; --i) {                                                 // top
                int a = gid(i, ny - 1), b = gid(i - 1, ny - 1);
                add(a, b, (nt[a] == 2 && nt[b] == 2) ? 2 : 1);
            }
            for (int j = ny - 1; j > 0; --j) add(gid(0, j), gid(0, j - 1), 1);                // left
        }
        std::vector<fvm_bc> bcs = {fvm_bc{1, 3, 0.0, 0.0, 0.0}, fvm_bc{2, 1, 0.0, 0.0, 0.0}};
        finish_problem(out, 2, coords, en, ez, eK, bn, be, bt, nt, zones, bcs, nx, ny, 1);
        out->water_table = 0.0;
        out->t_end = 86400.0;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_problem_richards3d(int nx, int ny, int nz, double Lx, double Ly, double Lz,
                                      double jitter, uint64_t seed, double ln_var, double cxl,
                                      double cyl, double czl, double Kg, fvm_problem* out) {
    try {
        if (nx < 1 || ny < 1 || nz < 1 || !out || jitter < 0.0 || jitter >= 0.2)
            throw Error("fvm_problem_richards3d: bad arguments");
        int Nx = nx + 1, Ny = ny + 1, Nz = nz + 1;
        size_t N = (size_t)Nx * Ny * Nz;
        if (N > (size_t)INT32_MAX / 8) throw Error("mesh too large");
        double hx = Lx / nx, hy = Ly / ny, hz = Lz / nz;
        Rng rng(seed);
        std::vector<double> g(3 * N);
        for (int k = 0; k < Nz; ++k)
            for (int j = 0; j < Ny; ++j)
                for (int i = 0; i < Nx; ++i) {
                    double dx = (2.0 * rng.uniform() - 1.0) * jitter * hx;
                    double dy = (2.0 * rng.uniform() - 1.0) * jitter * hy;
                    double dz = (2.0 * rng.uniform() - 1.0) * jitter * hz;
                    if (i == 0 || i == nx) dx = 0.0;
                    if (j == 0 || j == ny) dy = 0.0;
                    if (k == 0 || k == nz) dz = 0.0;
                    size_t q = i + (size_t)Nx * (j + (size_t)Ny * k);
                    g[3 * q] = i * hx + dx; g[3 * q + 1] = j * hy + dy; g[3 * q + 2] = k * hz + dz;
                }
        // tile so that one tile holds roughly 1.3k nodes (8x8 columns for the
        // 21-node columns of the benchmark box)
        int tile = std::max(2, (int)std::lround(std::sqrt(1344.0 / Nz)));
        std::vector<int> perm = tiled_order(Nx, Ny, Nz, tile, tile);
        std::vector<double> coords(3 * N);
        for (size_t q = 0; q < N; ++q)
            for (int d = 0; d < 3; ++d) coords[3 * (size_t)perm[q] + d] = g[3 * q + d];
        auto nid = [&](int i, int j, int k) { return perm[i + (size_t)Nx * (j + (size_t)Ny * k)]; };
        // Kuhn split: 6 tets per cell around the (0,0,0)-(1,1,1) diagonal,
        // conforming across cells because every cell uses the same diagonal
        static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        std::vector<int> corder = tiled_order(nx, ny, nz, tile, tile);
        std::vector<int> cells((size_t)nx * ny * nz);
        for (size_t c = 0; c < cells.size(); ++c) cells[corder[c]] = (int)c;
        std::vector<double> fK = gaussian_field(nx, ny, nz, hx, hy, hz, ln_var, cxl, cyl, czl, seed ^ 0x5A5A5A5Aull);
        size_t T = cells.size() * 6;
        std::vector<int> en; en.reserve(4 * T);
        std::vector<int> ez(T, 0);
        std::vector<double> eK(T);
        std::vector<int> bn, be, bt;
        auto on_plane = [&](const int (*ijk)[3], int a, int b, int c, int& tag) -> bool {
            // boundary face if the three nodes share a boundary plane
            for (int d = 0; d < 3; ++d) {
                int lim[2] = {0, d == 0 ? nx : (d == 1 ? ny : nz)};
                for (int s = 0; s < 2; ++s)
                    if (ijk[a][d] == lim[s] && ijk[b][d] == lim[s] && ijk[c][d] == lim[s]) {
                        if (d == 2 && s == 1) tag = 2;          // top: recharge
                        else if (d == 0 && s == 0) tag = 3;     // x = 0: fixed head
                        else tag = 1;                           // no flow
                        return true;
                    }
            }
            return false;
        };
        size_t e = 0;
        for (int c : cells) {
            int ci = c % nx, cj = (c / nx) % ny, ck = c / (nx * ny);
            for (int p = 0; p < 6; ++p, ++e) {
                int ijk[4][3];
                ijk[0][0] = ci; ijk[0][1] = cj; ijk[0][2] = ck;
                for (int s = 1; s <= 2; ++s) {
                    for (int d = 0; d < 3; ++d) ijk[s][d] = ijk[s - 1][d];
                    ijk[s][perms[p][s - 1]] += 1;
                }
                ijk[3][0] = ci + 1; ijk[3][1] = cj + 1; ijk[3][2] = ck + 1;
                int v[4];
                for (int s = 0; s < 4; ++s) v[s] = nid(ijk[s][0], ijk[s][1], ijk[s][2]);
                // positive orientation
                const double *A = &coords[3 * (size_t)v[0]], *B = &coords[3 * (size_t)v[1]],
                             *C = &coords[3 * (size_t)v[2]], *D = &coords[3 * (size_t)v[3]];
                double u[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
                double w[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
                double r[3] = {D[0] - A[0], D[1] - A[1], D[2] - A[2]};
                double vol = u[0] * (w[1] * r[2] - w[2] * r[1]) - u[1] * (w[0] * r[2] - w[2] * r[0]) + u[2] * (w[0] * r[1] - w[1] * r[0]);
                if (vol < 0) { std::swap(v[2], v[3]); for (int d = 0; d < 3; ++d) std::swap(ijk[2][d], ijk[3][d]); vol = -vol; }
                if (vol <= 1e-12 * hx * hy * hz) throw Error("jitter too large: degenerate tetrahedron");
                for (int s = 0; s < 4; ++s) en.push_back(v[s]);
                eK[e] = Kg * std::exp(fK[ci + (size_t)nx * (cj + (size_t)ny * ck)]);
                static const int fl[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
                for (auto& f : fl) {
                    int tag;
                    if (on_plane(ijk, f[0], f[1], f[2], tag)) {
                        bn.push_back(v[f[0]]); bn.push_back(v[f[1]]); bn.push_back(v[f[2]]);
                        be.push_back((int)e); bt.push_back(tag);
                    }
                }
            }
        }
        std::vector<int> nt(N, 0);
        for (int k = 0; k < Nz; ++k)
            for (int j = 0; j < Ny; ++j) nt[nid(0, j, k)] = 3;
        double water_table = 0.5 * Lz;
        std::vector<fvm_zone> zones = {fvm_zone{Kg, Kg, Kg, 0.42, 2.0, 1.8, 0.06 / 0.42}};
        std::vector<fvm_bc> bcs = {fvm_bc{1, 3, 0.0, 0.0, 0.0}, fvm_bc{2, 3, -1e-7, 0.0, 0.0},
                                   fvm_bc{3, 4, 0.0, water_table, 0.0}};
        finish_problem(out, 3, coords, en, ez, eK, bn, be, bt, nt, zones, bcs, Nx, Ny, Nz);
        out->water_table = water_table;
        out->t_end = 30.0 * 86400.0;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

// Ensemble of independent 2D problems as one disjoint mesh: member m has
// N_m ~ U[nmin, nmax] nodes on the 10 m x 5 m box (nx ~ sqrt(2 N_m)), its own
// jitter seed and its own lognormal Ks field (ln-variance ~ U[0.5, 2],
// correlation length ~ U[0.5, 3] m), the two soil layers and the boundary
// conditions of the 2D problem.  Node, element and boundary-face ids of the
// members are offset so that member m owns nodes [member_ptr[m],
// member_ptr[m+1]); elements and faces never couple two members.
extern "C" int fvm_problem_ensemble2d(int n_members, int nmin, int nmax, uint64_t seed, fvm_problem* out,
                                      int* member_ptr) {
    try {
        if (n_members < 1 || nmin < 16 || nmax < nmin || !out || !member_ptr)
            throw Error("fvm_problem_ensemble2d: bad arguments");
        Rng rng(seed);
        std::vector<double> coords, eK;
        std::vector<int> en, ez, bn, be, bt, nt;
        std::vector<fvm_zone> zones;
        std::vector<fvm_bc> bcs;
        member_ptr[0] = 0;
        for (int m = 0; m < n_members; ++m) {
            const double target = nmin + (nmax - nmin) * rng.uniform();
            const int nx = std::max(3, (int)std::lround(std::sqrt(2.0 * target)));
            const int ny = std::max(3, (int)std::lround(target / nx));
            const double ln_var = 0.5 + 1.5 * rng.uniform();
            const double corr = 0.5 + 2.5 * rng.uniform();
            const uint64_t ms = rng.next();
            fvm_problem pm;
            if (fvm_problem_richards2d(nx, ny, 10.0, 5.0, 0.2, ms, ln_var, corr, &pm) != 0)
                throw Error("fvm_problem_ensemble2d: member generation failed");
            const int n0 = (int)(coords.size() / 3), e0 = (int)ez.size();
            const fvm_mesh& mm = pm.mesh;
            coords.insert(coords.end(), mm.coords, mm.coords + 3 * (size_t)mm.n_nodes);
            for (int q = 0; q < 3 * mm.n_elements; ++q) en.push_back(mm.elem_nodes[q] + n0);
            ez.insert(ez.end(), mm.elem_zone, mm.elem_zone + mm.n_elements);
            if (mm.elem_K) eK.insert(eK.end(), mm.elem_K, mm.elem_K + mm.n_elements);
            else for (int e = 0; e < mm.n_elements; ++e) eK.push_back(pm.zones[mm.elem_zone[e]].Kxx);
            for (int q = 0; q < 2 * mm.n_bfaces; ++q) bn.push_back(mm.bface_nodes[q] + n0);
            for (int q = 0; q < mm.n_bfaces; ++q) be.push_back(mm.bface_elem[q] + e0);
            bt.insert(bt.end(), mm.bface_tag, mm.bface_tag + mm.n_bfaces);
            nt.insert(nt.end(), mm.node_tag, mm.node_tag + mm.n_nodes);
            if (m == 0) {
                zones.assign(pm.zones, pm.zones + pm.phys.n_zones);
                bcs.assign(pm.bcs, pm.bcs + pm.phys.n_bcs);
            }
            member_ptr[m + 1] = n0 + mm.n_nodes;
            fvm_problem_free(&pm);
        }
        finish_problem(out, 2, coords, en, ez, eK, bn, be, bt, nt, zones, bcs, (int)(coords.size() / 3), 1, 1);
        out->water_table = 0.0;
        out->t_end = 86400.0;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" void fvm_problem_free(fvm_problem* p) {
    if (!p) return;
    std::free(p->coords); std::free(p->elem_nodes); std::free(p->elem_zone); std::free(p->elem_K);
    std::free(p->bface_nodes); std::free(p->bface_elem); std::free(p->bface_tag);
    std::free(p->node_tag); std::free(p->zones); std::free(p->bcs); std::free(p->grid_dims);
    std::memset(p, 0, sizeof(*p));
}
