// FP64 CPU ORACLE for the FVMPor Richards hot path — test infrastructure.
//
// This file restates, on the host, the reference's own algorithm for the
// residual F(t, y, y'), the frozen upwinding, the coloured finite-
// difference Jacobian, ILU(0), GMRES and the BDF time step.  It exists to
// check the B200 kernels and to be timed as the CPU baseline; nothing in the
// product calls it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline use it.
//
// Parity status: the reference cannot be built here (SUNDIALS IDAS, MKL,
// minlin, Boost, MPI and ParMETIS are absent) and ships no tests or golden
// vectors for this path, so the oracle is pinned by known-answer tests
// (closed-form van Genuchten values, exact linear fields, closed control
// volumes, mass balance) and a loose comparison against the reference's
// stored run output, not by executing the reference.
//
// Data flow follows the reference step by step:
//   geometry   src/fvm/mesh.cpp:369-441 (element edge/face tables), :786-1156
//              (CV faces, SCV volumes, boundary CV faces, face sort by
//              (edge, element)), :1453-1543 (back faces, triangle_volume,
//              pyramid_volume), include/fvm/impl/mesh/cvface_shape.h:49-107,
//              cvface_inline.h:110-175 (area-weighted normal back -> front)
//   set-up     examples/fvmporMinlin/fvmpor.h:347-644 (zones, SCV weights,
//              Dirichlet rows), :948-1124 (shape-gradient, flux-limiter and
//              CV-flux CSR matrices), shape.cpp:27-60, :98-135
//   residual   fvmpor_ODE_impl.cpp:62-116, fvmpor.h:280-344 (saturation, CPU
//              branch), :647-759 (faces, fluxes), :875-945 (psk, ahh)
//   upwinding  fvmpor_ODE_impl.cpp:118-141, fvmpor.h:762-795
//   Jacobian   preconditioner_dss.cpp:21-142 (pattern, distance-2
//              colouring), :284-373 (shift and per-colour residuals)
//   ILU(0)     decomp/ILU.c:12-115, :133-223
//   GMRES      decomp/gmres.c:26-201, :412-511 (modified Gram-Schmidt), left
//              preconditioned and ewt-scaled as IDAS SPGMR runs it
// The adaptive time loop (orc_integrate) instantiates the product's BDF
// controller template (fvmpor_b200/csrc/bdf_controller.hpp), so oracle and GPU
// adaptive runs differ only in the kernels.  The step-sequence replay
// (orc_replay) does NOT use it: it restates the fixed-leading-coefficient BDF
// step independently, as Lagrange interpolation through the stored solution
// values, so a replay comparison also checks the controller's formulas.
#include "../include/fvmpor_b200.h"
#include "../fvmpor_b200/csrc/bdf_controller.hpp"

#include <omp.h>

#include <algorithm>
#include <cassert>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace orc {

struct P3 {
    double x = 0, y = 0, z = 0;
};
static inline P3 operator+(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline P3 operator-(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline P3 operator*(double s, P3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline P3 operator/(P3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
static inline double dot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline P3 cross(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static inline double norm(P3 a) { return std::sqrt(dot(a, a)); }

// CVFace_shape (cvface_shape.h)
struct Shape {
    P3 p[4];
    int n = 0;
    double area() const {
        if (n == 2) return norm(p[1] - p[0]);
        return (norm(cross(p[1] - p[0], p[3] - p[0])) + norm(cross(p[1] - p[2], p[3] - p[2]))) / 2.0;
    }
    P3 normal() const {
        P3 r = n == 2 ? cross(p[1] - p[0], P3{0, 0, 1}) : cross(p[1] - p[0], p[3] - p[0]);
        return r / norm(r);
    }
};

static double triangle_volume(P3 p1, P3 p2, P3 p3) {
    P3 v1 = p1 - p2, v2 = p1 - p3;
    double a = dot(v1, v1), b = dot(v2, v2), c = dot(v1, v2);
    return std::sqrt(a * b - c * c) / 2.0;
}

// |area * height / 3|, height = distance from the apex to the plane through
// points 0, 1, 3 of the face (mesh.cpp pyramid_volume)
static double pyramid_volume(const Shape& f, P3 apex) {
    P3 nn = f.normal();
    double height = dot(apex - f.p[0], nn);
    return std::fabs(f.area() * height / 3.0);
}

struct CSR {
    std::vector<int> ia, ja;
    std::vector<double> a;
    int rows() const { return (int)ia.size() - 1; }
    // InterpolationMatrix::matvec (include/util/interpolation.h:83-125)
    void matvec(const double* x, double* y) const {
        int n = rows();
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int p = ia[i]; p < ia[i + 1]; ++p) s += a[p] * x[ja[p]];
            y[i] = s;
        }
    }
};

struct Zone {
    double Kxx, Kyy, Kzz, phi, alphaVG, nVG, mVG, S_r;
};

struct Oracle {
    int dim = 0, N = 0, T = 0, npe = 0, nfe = 0;
    double rho0 = 1000.0;
    std::vector<P3> X;
    std::vector<int> en;       // [T][npe]
    std::vector<int> ezone;
    std::vector<double> eKx, eKy, eKz;
    std::vector<Zone> zones;
    std::map<int, fvm_bc> bcs;
    // edges
    int E = 0;
    std::vector<int> edge_front, edge_back;
    // CV faces: interior first (sorted by (edge, element)), then boundary
    int Fi = 0, Fall = 0;
    std::vector<int> cf_elem, cf_front, cf_back, cf_edge, cf_btag;
    std::vector<double> cf_area;
    std::vector<P3> cf_normal;     // area-weighted
    std::vector<double> cvvol;     // control volumes
    std::vector<std::vector<std::pair<int, double>>> scv;   // per node: (element, scv volume), ascending element
    // set-up products
    CSR Sx, Sy, Sz, flux_lim, cvflux;
    std::vector<int> zone_tags;                   // zones present, ascending
    std::vector<std::vector<int>> index_scv;      // per zone: node list
    std::vector<std::vector<double>> weight_scv;  // per zone: SCV volume fraction
    std::vector<int> is_dirichlet;                // per node: tag or 0
    std::vector<int> dirichlet_nodes;
    std::vector<double> h_dirichlet;
    std::vector<double> Kfx, Kfy, Kfz;            // negated K per interior face
    std::vector<double> w_front, w_back;          // per edge
    std::vector<double> qdotn_bnd_const;          // per boundary face (type 3)
    // work
    std::vector<double> h, hp, gx, gy, gz, phi_vec, dSw_vec, ahh, krw_f, qdotn, Mflux;
    long n_res = 0;
    // time split of the integrations and replays (seconds): Newton residuals
    // (with the begin-step evaluation), J*v, finite-difference Jacobian, ILU
    // factor, preconditioner apply, Krylov orthogonalisation and least
    // squares, whole run; and their work counters: Newton residuals, J*v
    // products, set-ups, applies, Krylov iterations, Newton iterations,
    // steps (the reference prints the same split, examples/fvmporMinlin/
    // fvmpor_ODE.cpp:233-245)
    double tm[7] = {};
    long cnt[7] = {};
    std::vector<fvm_step_record> last_trace;
    // preconditioner
    bool pat_built = false;
    std::vector<int> jrow, jcol, colour;
    int ncol = 0;
    std::vector<double> J;
    std::vector<int> bstart;
    // ILU(0) of the block-diagonal part, each block's rows in colour order:
    // factor position q is global row frow[q]; fptr/fcol/fdiag index
    // positions, fsrc the source entry of J
    std::vector<int> frow, fptr, fcol, fsrc, fdiag;
    std::vector<double> LU;
    // Schur interface coupling (decomp/schur.c:887-987, 1407-1636).  < 0:
    // off (block-Jacobi ILU(0)).  >= 0: every block orders its interior
    // rows (no coupling outside the block) before its interface rows, each
    // group in colour order, and the apply iterates the interface system
    // that many times against the other blocks' interface values.
    // fifc[b]: first interface position of block b; optr/ocol/osrc: the
    // off-block entries of each factor position (global column, J entry),
    // in J's column order.
    int schur_iters = -1;
    std::vector<int> fifc, optr, ocol, osrc;

    void build(const fvm_mesh* m, const fvm_physics* ph);
    void residual(double t, const double* y, const double* yp, double* res);
    void preprocess_evaluation(double t, const double* y, const double* yp);
    void residual_evaluation(double* res);
    void begin_step(double t, const double* y, const double* yp);
    void jv(double t, double cj, const double* y, const double* yp, const double* F0, const double* v,
            double sigma, double* Jv);
    void psetup(double t, double cj, double hh, const double* y, const double* yp, const double* F0,
                const double* ewt, int nb);
    int ilu_factor();
    // psetup + ilu_factor with the time split booked
    int timed_psetup(double t, double cj, double hh, const double* y, const double* yp, const double* F0,
                     const double* ewt, int nb) {
        const double a = omp_get_wtime();
        psetup(t, cj, hh, y, yp, F0, ewt, nb);
        const double b = omp_get_wtime();
        const int r = ilu_factor();
        tm[2] += b - a;
        tm[3] += omp_get_wtime() - b;
        cnt[2]++;
        return r;
    }
    void psolve(const double* r, double* z) const;
    int gmres(double cj, const double* y, const double* yp, const double* F0, const double* ewt,
              const double* b, double* x, int m, int max_restarts, double tol, int* iters,
              double* rn, long* njv, long* nps);
};

// ---------------------------------------------------------------- geometry
void Oracle::build(const fvm_mesh* m, const fvm_physics* ph) {
    dim = m->dim;
    N = m->n_nodes;
    T = m->n_elements;
    npe = dim + 1;
    nfe = dim == 2 ? 3 : 6;
    rho0 = ph->rho0;
    X.resize(N);
    for (int i = 0; i < N; ++i) X[i] = P3{m->coords[3 * i], m->coords[3 * i + 1], m->coords[3 * i + 2]};
    en.assign(m->elem_nodes, m->elem_nodes + (size_t)T * npe);
    ezone.assign(m->elem_zone, m->elem_zone + T);
    zones.resize(ph->n_zones);
    for (int z = 0; z < ph->n_zones; ++z) {
        const fvm_zone& s = ph->zones[z];
        zones[z] = Zone{s.Kxx, s.Kyy, s.Kzz, s.phi, s.alphaVG, s.nVG, 1.0 - 1.0 / s.nVG, s.S_r};
    }
    eKx.resize(T); eKy.resize(T); eKz.resize(T);
    for (int e = 0; e < T; ++e) {
        const Zone& Z = zones[ezone[e]];
        eKx[e] = m->elem_K ? m->elem_K[e] : Z.Kxx;
        eKy[e] = m->elem_K ? m->elem_K[e] : Z.Kyy;
        eKz[e] = m->elem_K ? m->elem_K[e] : Z.Kzz;
    }
    for (int b = 0; b < ph->n_bcs; ++b) bcs[ph->bcs[b].tag] = ph->bcs[b];

    // element edge and face tables (mesh.cpp:383-441)
    static const int tri_e[3][2] = {{0, 1}, {1, 2}, {2, 0}};
    static const int tet_e[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
    static const int tet_f[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    static const int tet_fe[4][3] = {{0, 1, 2}, {0, 4, 3}, {2, 5, 3}, {1, 5, 4}};
    static const int tri_f[3][2] = {{0, 1}, {1, 2}, {2, 0}};
    auto ledge = [&](int f, int s) { return dim == 2 ? tri_e[f][s] : tet_e[f][s]; };

    // edges: first encounter fixes front/back; ids = rank of (min, max)
    std::map<std::pair<int, int>, std::pair<int, int>> emap;   // key -> (front, back)
    for (int e = 0; e < T; ++e)
        for (int f = 0; f < nfe; ++f) {
            int a = en[(size_t)e * npe + ledge(f, 0)], b = en[(size_t)e * npe + ledge(f, 1)];
            auto key = std::make_pair(std::min(a, b), std::max(a, b));
            if (!emap.count(key)) emap[key] = std::make_pair(a, b);
        }
    E = (int)emap.size();
    std::map<std::pair<int, int>, int> eid;
    edge_front.resize(E);
    edge_back.resize(E);
    {
        int id = 0;
        for (auto& kv : emap) {
            eid[kv.first] = id;
            edge_front[id] = kv.second.first;
            edge_back[id] = kv.second.second;
            ++id;
        }
    }
    auto edge_of = [&](int a, int b) { return eid.at(std::make_pair(std::min(a, b), std::max(a, b))); };
    std::vector<P3> ecent(T);
    for (int e = 0; e < T; ++e) {
        P3 c;
        for (int k = 0; k < npe; ++k) c = c + X[en[(size_t)e * npe + k]];
        ecent[e] = c / (double)npe;
    }

    // boundary faces keyed by their sorted nodes
    std::map<std::vector<int>, int> btag;
    for (int b = 0; b < m->n_bfaces; ++b) {
        std::vector<int> key(m->bface_nodes + (size_t)b * dim, m->bface_nodes + (size_t)(b + 1) * dim);
        std::sort(key.begin(), key.end());
        btag[key] = m->bface_tag[b];
    }

    // ---- interior CV faces and SCV volumes
    struct CF {
        int edge, elem, front, back;
        double area;
        P3 normal;
    };
    std::vector<CF> cfs;
    cfs.reserve((size_t)T * nfe);
    std::vector<std::vector<double>> scvvol(T, std::vector<double>(npe, 0.0));
    for (int e = 0; e < T; ++e) {
        const int* v = &en[(size_t)e * npe];
        if (dim == 2) {
            double orient = (X[v[1]].x - X[v[0]].x) * (X[v[2]].y - X[v[0]].y) - (X[v[1]].y - X[v[0]].y) * (X[v[2]].x - X[v[0]].x);
            if (!(orient > 0)) throw std::runtime_error("oracle: triangles must be counter-clockwise");
        }
        for (int f = 0; f < nfe; ++f) {
            int la = ledge(f, 0), lb = ledge(f, 1);
            int eg = edge_of(v[la], v[lb]);
            int front = edge_front[eg], back = edge_back[eg];
            int lfront = v[la] == front ? la : lb, lback = v[la] == front ? lb : la;
            P3 mid = (X[front] + X[back]) / 2.0;
            Shape q;
            Shape bf1, bf2;
            if (dim == 3) {
                // the two element faces containing the edge (faces_from_edge)
                int f1 = -1, f2 = -1;
                for (int ff = 0; ff < 4; ++ff)
                    for (int j = 0; j < 3; ++j)
                        if (tet_fe[ff][j] == f) { if (f1 < 0) f1 = ff; f2 = ff; }
                auto fcent = [&](int ff) {
                    return (X[v[tet_f[ff][0]]] + X[v[tet_f[ff][1]]] + X[v[tet_f[ff][2]]]) / 3.0;
                };
                q.n = 4;
                q.p[0] = mid; q.p[1] = fcent(f1); q.p[2] = ecent[e]; q.p[3] = fcent(f2);
                // back faces of the two SCVs (make_back_faces): the element face
                // holding the node's two other edges
                auto backface = [&](int ln) {
                    int oe[2], cnt = 0;
                    for (int j = 0; j < 6 && cnt < 2; ++j)
                        if (j != f && (tet_e[j][0] == ln || tet_e[j][1] == ln)) oe[cnt++] = j;
                    // second edge: the last match when scanning down (other_edges_for_node)
                    for (int j = 5; j >= 0; --j)
                        if (j != f && (tet_e[j][0] == ln || tet_e[j][1] == ln)) { oe[1] = j; break; }
                    int fid = -1;
                    for (int ff = 0; ff < 4 && fid < 0; ++ff) {
                        bool h1 = false, h2 = false;
                        for (int j = 0; j < 3; ++j) { h1 |= tet_fe[ff][j] == oe[0]; h2 |= tet_fe[ff][j] == oe[1]; }
                        if (h1 && h2) fid = ff;
                    }
                    Shape s;
                    s.n = 4;
                    s.p[0] = X[v[ln]];
                    s.p[1] = (X[v[tet_e[oe[0]][0]]] + X[v[tet_e[oe[0]][1]]]) / 2.0;
                    s.p[2] = fcent(fid);
                    s.p[3] = (X[v[tet_e[oe[1]][0]]] + X[v[tet_e[oe[1]][1]]]) / 2.0;
                    return s;
                };
                bf1 = backface(lfront);
                bf2 = backface(lback);
                P3 p1 = (ecent[e] + X[front]) / 2.0;
                scvvol[e][lfront] += pyramid_volume(q, p1);
                scvvol[e][lfront] += pyramid_volume(bf1, p1);
                P3 p2 = (ecent[e] + X[back]) / 2.0;
                scvvol[e][lback] += pyramid_volume(q, p2);
                scvvol[e][lback] += pyramid_volume(bf2, p2);
            } else {
                q.n = 2;
                q.p[0] = mid;
                q.p[1] = ecent[e];
                scvvol[e][lfront] += triangle_volume(ecent[e], mid, X[front]);
                scvvol[e][lback] += triangle_volume(ecent[e], mid, X[back]);
            }
            CF cf;
            cf.edge = eg;
            cf.elem = e;
            cf.front = front;
            cf.back = back;
            cf.area = q.area();
            P3 nn = q.normal();
            if (dot(nn, X[front] - X[back]) < 0.0) nn = -1.0 * nn;
            cf.normal = cf.area * nn;
            cfs.push_back(cf);
        }
    }
    // sort interior CV faces by (edge, element) (mesh.cpp:802-825)
    std::stable_sort(cfs.begin(), cfs.end(), [](const CF& a, const CF& b) {
        if (a.edge != b.edge) return a.edge < b.edge;
        return a.elem < b.elem;
    });
    Fi = (int)cfs.size();
    // boundary CV faces in element / face / node order (mesh.cpp:1046-1156)
    struct BF {
        int elem, node, tag;
        double area;
    };
    std::vector<BF> bfs;
    for (int e = 0; e < T; ++e) {
        const int* v = &en[(size_t)e * npe];
        int nf = dim == 2 ? 3 : 4;
        for (int ff = 0; ff < nf; ++ff) {
            std::vector<int> fn;
            if (dim == 2) fn = {v[tri_f[ff][0]], v[tri_f[ff][1]]};
            else fn = {v[tet_f[ff][0]], v[tet_f[ff][1]], v[tet_f[ff][2]]};
            std::vector<int> key = fn;
            std::sort(key.begin(), key.end());
            auto it = btag.find(key);
            if (it == btag.end()) continue;
            P3 fc;
            for (int n : fn) fc = fc + X[n];
            fc = fc / (double)fn.size();
            for (size_t k = 0; k < fn.size(); ++k) {
                Shape q;
                if (dim == 2) {
                    q.n = 2;
                    q.p[0] = X[fn[k]];
                    q.p[1] = fc;
                } else {
                    // the face's two edges at node k (edges_from_node)
                    int a = fn[(k + 1) % 3], b = fn[(k + 2) % 3];
                    q.n = 4;
                    q.p[0] = X[fn[k]];
                    q.p[1] = (X[fn[k]] + X[a]) / 2.0;
                    q.p[2] = fc;
                    q.p[3] = (X[fn[k]] + X[b]) / 2.0;
                }
                bfs.push_back(BF{e, fn[k], it->second, q.area()});
            }
        }
    }
    Fall = Fi + (int)bfs.size();
    cf_elem.resize(Fall); cf_front.resize(Fall); cf_back.resize(Fall); cf_edge.resize(Fall);
    cf_btag.resize(Fall); cf_area.resize(Fall); cf_normal.resize(Fi);
    for (int i = 0; i < Fi; ++i) {
        cf_elem[i] = cfs[i].elem; cf_front[i] = cfs[i].front; cf_back[i] = cfs[i].back;
        cf_edge[i] = cfs[i].edge; cf_btag[i] = 0; cf_area[i] = cfs[i].area; cf_normal[i] = cfs[i].normal;
    }
    for (size_t b = 0; b < bfs.size(); ++b) {
        int i = Fi + (int)b;
        cf_elem[i] = bfs[b].elem; cf_front[i] = -1; cf_back[i] = bfs[b].node; cf_edge[i] = -1;
        cf_btag[i] = bfs[b].tag; cf_area[i] = bfs[b].area;
    }
    // control volumes: sum of SCVs in ascending element order
    scv.assign(N, {});
    for (int e = 0; e < T; ++e)
        for (int k = 0; k < npe; ++k) scv[en[(size_t)e * npe + k]].push_back({e, scvvol[e][k]});
    cvvol.assign(N, 0.0);
    for (int i = 0; i < N; ++i) {
        if (scv[i].empty()) throw std::runtime_error("oracle: node without element");
        for (auto& s : scv[i]) cvvol[i] += s.second;
    }

    // ---- zones, SCV weights (fvmpor.h:455-498)
    std::set<int> zs(ezone.begin(), ezone.end());
    zone_tags.assign(zs.begin(), zs.end());
    int nz = (int)zone_tags.size();
    std::map<int, int> zmap;
    for (int z = 0; z < nz; ++z) zmap[zone_tags[z]] = z;
    index_scv.assign(nz, {});
    weight_scv.assign(nz, {});
    for (int i = 0; i < N; ++i) {
        std::vector<double> w(nz, 0.0);
        std::vector<int> cnt(nz, 0);
        for (auto& s : scv[i]) {
            int z = zmap[ezone[s.first]];
            w[z] += s.second / cvvol[i];
            cnt[z]++;
        }
        for (int z = 0; z < nz; ++z)
            if (cnt[z]) { weight_scv[z].push_back(w[z]); index_scv[z].push_back(i); }
    }
    // ---- Dirichlet rows (fvmpor.h:404-451)
    is_dirichlet.assign(N, 0);
    for (int i = 0; i < N; ++i) {
        int tag = m->node_tag[i];
        if (tag && bcs.count(tag) && (bcs[tag].type == 1 || bcs[tag].type == 4)) is_dirichlet[i] = tag;
    }
    dirichlet_nodes.clear();
    h_dirichlet.clear();
    for (int i = 0; i < N; ++i)
        if (is_dirichlet[i]) {
            const fvm_bc& bc = bcs[is_dirichlet[i]];
            double el = dim == 2 ? X[i].y : X[i].z;
            dirichlet_nodes.push_back(i);
            h_dirichlet.push_back(bc.type == 1 ? bc.value : (1.0 + bc.eta) * (bc.b - el));
        }

    // ---- shape-gradient CSR over interior CV faces (fvmpor.h:948-1024)
    auto shape_grads = [&](int e, std::vector<P3>& g) {
        const int* v = &en[(size_t)e * npe];
        g.assign(npe, P3{});
        if (dim == 2) {
            double A = 0.0;
            for (int k = 0; k < 3; ++k) A += scvvol[e][k];
            double x0 = X[v[0]].x, x1 = X[v[1]].x, x2 = X[v[2]].x;
            double y0 = X[v[0]].y, y1 = X[v[1]].y, y2 = X[v[2]].y;
            double dNdx[3] = {(y1 - y2) / (2 * A), (y2 - y0) / (2 * A), (y0 - y1) / (2 * A)};
            double dNdy[3] = {(x2 - x1) / (2 * A), (x0 - x2) / (2 * A), (x1 - x0) / (2 * A)};
            for (int k = 0; k < 3; ++k) g[k] = P3{dNdx[k], dNdy[k], 0.0};
        } else {
            auto det3 = [](double a11, double a12, double a13, double a21, double a22, double a23,
                           double a31, double a32, double a33) {
                return a11 * a22 * a33 - a11 * a23 * a32 - a21 * a12 * a33 + a21 * a13 * a32 + a31 * a12 * a23 - a31 * a13 * a22;
            };
            double Nxi[] = {-1.0, 1.0, 0.0, 0.0}, Net[] = {-1.0, 0.0, 1.0, 0.0}, Nze[] = {-1.0, 0.0, 0.0, 1.0};
            double x_xi = 0, x_et = 0, x_ze = 0, y_xi = 0, y_et = 0, y_ze = 0, z_xi = 0, z_et = 0, z_ze = 0;
            for (int j = 0; j < 4; ++j) {
                P3 p = X[v[j]];
                x_xi += p.x * Nxi[j]; x_et += p.x * Net[j]; x_ze += p.x * Nze[j];
                y_xi += p.y * Nxi[j]; y_et += p.y * Net[j]; y_ze += p.y * Nze[j];
                z_xi += p.z * Nxi[j]; z_et += p.z * Net[j]; z_ze += p.z * Nze[j];
            }
            double del = det3(x_xi, y_xi, z_xi, x_et, y_et, z_et, x_ze, y_ze, z_ze);
            for (int j = 0; j < 4; ++j) {
                double dx = det3(Nxi[j], y_xi, z_xi, Net[j], y_et, z_et, Nze[j], y_ze, z_ze);
                double dy = det3(x_xi, Nxi[j], z_xi, x_et, Net[j], z_et, x_ze, Nze[j], z_ze);
                double dz = det3(x_xi, y_xi, Nxi[j], x_et, y_et, Net[j], x_ze, y_ze, Nze[j]);
                g[j] = P3{dx, dy, dz} / del;
            }
        }
    };
    Sx.ia.assign(Fi + 1, 0);
    for (int i = 0; i < Fi; ++i) Sx.ia[i + 1] = Sx.ia[i] + npe;
    Sx.ja.resize((size_t)Fi * npe);
    Sx.a.resize(Sx.ja.size());
    Sy = Sx;
    Sz = Sx;
    {
        std::vector<P3> g;
        for (int i = 0; i < Fi; ++i) {
            int e = cf_elem[i];
            shape_grads(e, g);
            std::vector<std::pair<int, int>> idx(npe);
            for (int k = 0; k < npe; ++k) idx[k] = {en[(size_t)e * npe + k], k};
            std::sort(idx.begin(), idx.end());
            for (int k = 0; k < npe; ++k) {
                size_t p = (size_t)i * npe + k;
                Sx.ja[p] = Sy.ja[p] = Sz.ja[p] = idx[k].first;
                Sx.a[p] = g[idx[k].second].x;
                Sy.a[p] = g[idx[k].second].y;
                Sz.a[p] = g[idx[k].second].z;
            }
        }
    }
    // flux limiter: edges x faces, weight 1 / total face area (:1033-1071)
    {
        std::vector<std::vector<int>> edge_cvf(E);
        for (int i = 0; i < Fi; ++i) edge_cvf[cf_edge[i]].push_back(i);
        flux_lim.ia.assign(E + 1, 0);
        for (int g = 0; g < E; ++g) {
            double tot = 0.0;
            for (int f : edge_cvf[g]) tot += cf_area[f];
            for (int f : edge_cvf[g]) { flux_lim.ja.push_back(f); flux_lim.a.push_back(1.0 / tot); }
            flux_lim.ia[g + 1] = (int)flux_lim.ja.size();
        }
    }
    // CV flux: nodes x faces, -1/V on the back node, +1/V on the front
    // (:1079-1122), faces ascending per row
    {
        std::vector<std::vector<int>> nf(N);
        for (int f = 0; f < Fall; ++f) {
            nf[cf_back[f]].push_back(f);
            if (cf_front[f] >= 0) nf[cf_front[f]].push_back(f);
        }
        cvflux.ia.assign(N + 1, 0);
        for (int i = 0; i < N; ++i) {
            std::sort(nf[i].begin(), nf[i].end());
            double w = 1.0 / cvvol[i];
            for (int f : nf[i]) {
                cvflux.ja.push_back(f);
                cvflux.a.push_back(i == cf_back[f] ? -w : w);
            }
            cvflux.ia[i + 1] = (int)cvflux.ja.size();
        }
    }
    // negated face conductivities (:632-643)
    Kfx.resize(Fi); Kfy.resize(Fi); Kfz.resize(Fi);
    for (int i = 0; i < Fi; ++i) {
        int e = cf_elem[i];
        Kfx[i] = -eKx[e]; Kfy[i] = -eKy[e]; Kfz[i] = -eKz[e];
    }
    qdotn_bnd_const.assign(Fall - Fi, 0.0);
    for (int b = 0; b < Fall - Fi; ++b) {
        auto it = bcs.find(cf_btag[Fi + b]);
        if (it == bcs.end()) throw std::runtime_error("oracle: boundary tag without condition");
        if (it->second.type == 3) qdotn_bnd_const[b] = it->second.value * cf_area[Fi + b];
    }
    w_front.assign(E, 0.5);
    w_back.assign(E, 0.5);
    h.resize(N); hp.resize(N); gx.resize(Fi); gy.resize(Fi); gz.resize(Fi);
    phi_vec.resize(N); dSw_vec.resize(N); ahh.resize(N); krw_f.resize(Fi);
    qdotn.resize(Fall); Mflux.resize(Fall);
}

// saturation, CPU branch of fvmpor.h:302-343
static void saturation(const std::vector<double>& hh, const Zone& z, std::vector<double>& Sw,
                       std::vector<double>& dSw, std::vector<double>& krw) {
    size_t n = hh.size();
    Sw.resize(n); dSw.resize(n); krw.resize(n);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) {
        double d = -z.alphaVG * hh[i];
        d = std::pow(d, z.nVG);
        double s = d + 1.0;
        double k = -1.0;
        k /= s;
        d /= s;
        s = std::pow(s, -z.mVG);
        d *= s;
        d /= hh[i];
        d *= -(1 - z.S_r) * (z.nVG - 1);
        k += 1.0;
        k = std::pow(k, z.mVG);
        k -= 1.0;
        k = k * k;
        k *= std::sqrt(s);
        s *= (1 - z.S_r);
        s += z.S_r;
        if (hh[i] >= 0.0) { d = 0.0; s = 1.0; k = 1.0; }
        Sw[i] = s; dSw[i] = d; krw[i] = k;
    }
}

void Oracle::preprocess_evaluation(double t, const double* y, const double* yp) {
    (void)t;
    n_res++;
    std::copy(y, y + N, h.begin());
    std::copy(yp, yp + N, hp.begin());
    Sx.matvec(h.data(), gx.data());
    Sy.matvec(h.data(), gy.data());
    if (dim == 3) Sz.matvec(h.data(), gz.data());
    // process_volumes_psk (:875-928)
    std::fill(phi_vec.begin(), phi_vec.end(), 0.0);
    std::fill(dSw_vec.begin(), dSw_vec.end(), 0.0);
    std::vector<double> head, Sw, dSw, krw;
    // face -> per-zone scv index of its front / back nodes
    for (size_t z = 0; z < zone_tags.size(); ++z) {
        const Zone& Z = zones[zone_tags[z]];
        const std::vector<int>& idx = index_scv[z];
        head.resize(idx.size());
        for (size_t q = 0; q < idx.size(); ++q) head[q] = h[idx[q]];
        saturation(head, Z, Sw, dSw, krw);
        for (size_t q = 0; q < idx.size(); ++q) {
            phi_vec[idx[q]] += Z.phi * weight_scv[z][q];
            dSw_vec[idx[q]] += dSw[q] * weight_scv[z][q];
        }
        // krw at faces of this zone, upwinded through the edge weights
        std::vector<double> krw_node(N, 0.0);
        for (size_t q = 0; q < idx.size(); ++q) krw_node[idx[q]] = krw[q];
#pragma omp parallel for schedule(static)
        for (int f = 0; f < Fi; ++f) {
            if (ezone[cf_elem[f]] != zone_tags[z]) continue;
            int g = cf_edge[f];
            double v = krw_node[cf_front[f]] * w_front[g];
            v += krw_node[cf_back[f]] * w_back[g];
            krw_f[f] = v;
        }
    }
    // process_derivative_coefficients (:931-945)
    for (int i = 0; i < N; ++i) {
        double a = phi_vec[i] * dSw_vec[i];
        ahh[i] = a * rho0;
    }
    // process_fluxes (:682-759); rho at faces is rho0 (beta = 0)
#pragma omp parallel for schedule(static)
    for (int f = 0; f < Fi; ++f) {
        double qx = gx[f] * Kfx[f];
        double qy = gy[f];
        double qz = 0.0;
        if (dim == 2) {
            qy += 1.0;
        } else {
            qz = gz[f];
            qz += 1.0;
            qz *= Kfz[f];
        }
        qy *= Kfy[f];
        double qn = cf_normal[f].x * qx;
        qn += cf_normal[f].y * qy;
        if (dim == 3) qn += cf_normal[f].z * qz;
        qn *= krw_f[f];
        qdotn[f] = qn;
        Mflux[f] = rho0 * qn;
    }
    for (int b = 0; b < Fall - Fi; ++b) {
        qdotn[Fi + b] = qdotn_bnd_const[b];
        Mflux[Fi + b] = rho0 * qdotn[Fi + b];
    }
}

void Oracle::residual_evaluation(double* res) {
    cvflux.matvec(Mflux.data(), res);
    for (int i = 0; i < N; ++i) res[i] -= hp[i] * ahh[i];
    for (size_t d = 0; d < dirichlet_nodes.size(); ++d) {
        int i = dirichlet_nodes[d];
        res[i] = h_dirichlet[d];
        res[i] -= h[i];
    }
}

void Oracle::residual(double t, const double* y, const double* yp, double* res) {
    preprocess_evaluation(t, y, yp);
    residual_evaluation(res);
}

void Oracle::begin_step(double t, const double* y, const double* yp) {
    std::fill(w_front.begin(), w_front.end(), 0.5);
    std::fill(w_back.begin(), w_back.end(), 0.5);
    preprocess_evaluation(t, y, yp);
    std::vector<double> ef(E);
    flux_lim.matvec(qdotn.data(), ef.data());
    for (int g = 0; g < E; ++g) {
        if (ef[g] < 0.0) { w_front[g] = 1.0; w_back[g] = 0.0; }
        else { w_front[g] = 0.0; w_back[g] = 1.0; }
    }
}

void Oracle::jv(double t, double cj, const double* y, const double* yp, const double* F0,
                const double* v, double sigma, double* Jv) {
    std::vector<double> y2(N), yp2(N), F(N);
    for (int i = 0; i < N; ++i) {
        y2[i] = y[i] + sigma * v[i];
        yp2[i] = yp[i] + cj * (sigma * v[i]);
    }
    residual(t, y2.data(), yp2.data(), F.data());
    for (int i = 0; i < N; ++i) Jv[i] = (F[i] - F0[i]) / sigma;
}

// ---------------------------------------------------------------- preconditioner
void Oracle::psetup(double t, double cj, double hh, const double* y, const double* yp,
                    const double* F0, const double* ewt, int nb) {
    if (!pat_built) {
        // column_pattern (:107-142): all (i, j) sharing an element
        std::vector<std::set<int>> rows(N);
        for (int e = 0; e < T; ++e)
            for (int a = 0; a < npe; ++a)
                for (int b = 0; b < npe; ++b) rows[en[(size_t)e * npe + a]].insert(en[(size_t)e * npe + b]);
        jrow.assign(N + 1, 0);
        jcol.clear();
        for (int i = 0; i < N; ++i) {
            jcol.insert(jcol.end(), rows[i].begin(), rows[i].end());
            jrow[i + 1] = (int)jcol.size();
        }
        // sequential_vertex_colouring over dependent_columns (:36-94)
        colour.assign(N, N - 1);
        std::vector<int> mark(N, -1);
        int maxc = 0;
        for (int i = 0; i < N; ++i) {
            std::set<int> cols;
            for (int p = jrow[i]; p < jrow[i + 1]; ++p)
                for (int q = jrow[jcol[p]]; q < jrow[jcol[p] + 1]; ++q) cols.insert(jcol[q]);
            for (int j : cols) mark[colour[j]] = i;
            int c = 0;
            while (c < maxc && mark[c] == i) ++c;
            if (c == maxc) ++maxc;
            colour[i] = c;
        }
        ncol = maxc;
        J.assign(jcol.size(), 0.0);
        pat_built = true;
    }
    // shift (:322-329)
    double eps = std::sqrt(DBL_EPSILON);
    std::vector<double> shift(N), ys(N), yps(N), Fs(N);
    for (int j = 0; j < N; ++j) shift[j] = eps * std::max(std::fabs(y[j]), std::max(std::fabs(hh * yp[j]), 1.0 / ewt[j]));
    for (int c = 0; c < ncol; ++c) {
        for (int j = 0; j < N; ++j) {
            ys[j] = y[j];
            yps[j] = yp[j];
            if (colour[j] == c) { ys[j] += shift[j]; yps[j] += cj * shift[j]; }
        }
        residual(t, ys.data(), yps.data(), Fs.data());
        for (int i = 0; i < N; ++i)
            for (int p = jrow[i]; p < jrow[i + 1]; ++p)
                if (colour[jcol[p]] == c) J[p] = (Fs[i] - F0[i]) / shift[jcol[p]];
    }
    // blocks of contiguous rows (nb = 1: global ILU(0))
    if (nb < 1) nb = 1;
    bstart.resize(nb + 1);
    for (int b = 0; b <= nb; ++b) bstart[b] = (int)(((long)N * b) / nb);
}

// Colour order of the rows [r0, r1) of a block (offsets from r0): greedy
// colouring in natural order (smallest colour unused by an earlier coupled
// row of the block), then stable by colour.  The same rule as the device
// factor's set-up: rows of one colour are uncoupled, so each triangular
// sweep of a block has as many levels as colours.
//
// With interface_last (the Schur coupling), rows coupled to a node outside
// the block (interface rows) come after all interior rows: the sort key is
// (interface, colour), so each (group, colour) is still one level.
static std::vector<int> block_colour_order(const std::vector<int>& jrow, const std::vector<int>& jcol, int r0,
                                           int r1, bool interface_last = false, int* n_interior = nullptr) {
    const int nr = r1 - r0;
    std::vector<int> colour(nr, 0), ord(nr), key(nr);
    int nin = 0;
    for (int i = r0; i < r1; ++i) {
        std::vector<int> used;
        bool iface = false;
        for (int p = jrow[i]; p < jrow[i + 1]; ++p) {
            const int j = jcol[p];
            if (j >= r0 && j < i) used.push_back(colour[j - r0]);
            if (j < r0 || j >= r1) iface = true;
        }
        std::sort(used.begin(), used.end());
        int cc = 0;
        for (int u : used)
            if (u == cc) ++cc;
        colour[i - r0] = cc;
        key[i - r0] = interface_last && iface ? (1 << 20) + cc : cc;
        if (!iface) ++nin;
    }
    if (n_interior) *n_interior = interface_last ? nin : nr;
    for (int ii = 0; ii < nr; ++ii) ord[ii] = ii;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return key[a] < key[b]; });
    return ord;
}

// ILU(0) on the block-diagonal part (decomp/ILU.c:12-115, pivot of row i
// inverted after its elimination), each block in its colour order
int Oracle::ilu_factor() {
    int nb = (int)bstart.size() - 1;
    frow.assign(N, 0);
    fptr.assign(N + 1, 0);
    fdiag.assign(N, -1);
    fcol.clear();
    fsrc.clear();
    std::vector<std::pair<int, int>> ent;
    const bool schur = schur_iters >= 0;
    fifc.assign(nb, 0);
    optr.assign(N + 1, 0);
    ocol.clear();
    osrc.clear();
    for (int b = 0; b < nb; ++b) {
        const int r0 = bstart[b], r1 = bstart[b + 1];
        int nin = 0;
        const std::vector<int> ord = block_colour_order(jrow, jcol, r0, r1, schur, &nin);
        fifc[b] = r0 + nin;
        std::vector<int> linv(r1 - r0);
        for (int ii = 0; ii < r1 - r0; ++ii) linv[ord[ii]] = ii;
        for (int ii = 0; ii < r1 - r0; ++ii) {
            const int i = r0 + ord[ii], q = r0 + ii;
            frow[q] = i;
            ent.clear();
            for (int p = jrow[i]; p < jrow[i + 1]; ++p) {
                const int j = jcol[p];
                if (j >= r0 && j < r1) ent.emplace_back(r0 + linv[j - r0], p);
                else if (schur) { ocol.push_back(j); osrc.push_back(p); }
            }
            optr[q + 1] = (int)ocol.size();
            std::sort(ent.begin(), ent.end());
            for (auto& e : ent) {
                if (e.first == q) fdiag[q] = (int)fcol.size();
                fcol.push_back(e.first);
                fsrc.push_back(e.second);
            }
            fptr[q + 1] = (int)fcol.size();
        }
    }
    LU.resize(fcol.size());
    for (size_t p = 0; p < fcol.size(); ++p) LU[p] = J[fsrc[p]];
    int bad = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : bad)
    for (int b = 0; b < nb; ++b) {
        for (int i = bstart[b]; i < bstart[b + 1]; ++i) {
            for (int kk = fptr[i]; kk < fdiag[i]; ++kk) {
                int k = fcol[kk];
                LU[kk] *= LU[fdiag[k]];
                int kpos = fdiag[k] + 1;
                for (int jj = kk + 1; jj < fptr[i + 1]; ++jj) {
                    int j = fcol[jj];
                    while (kpos < fptr[k + 1] && fcol[kpos] < j) ++kpos;
                    if (kpos == fptr[k + 1]) break;
                    if (fcol[kpos] == j) LU[jj] -= LU[kk] * LU[kpos];
                }
            }
            double d = LU[fdiag[i]];
            if (d == 0.0 || !std::isfinite(d)) { bad++; d = 1.0; }
            LU[fdiag[i]] = 1.0 / d;
        }
    }
    return bad ? 1 : 0;
}

void Oracle::psolve(const double* r, double* z) const {
    int nb = (int)bstart.size() - 1;
    if (schur_iters >= 0) {
        // Schur coupling of the blocks through their interface rows
        // (precon_schur_apply, decomp/schur.c:1407-1636).  With each block's
        // factor ordered [interior B; interface S~] = [L_B 0; F~ L_S] [U_B E~;
        // 0 U_S], S~ = L_S U_S is the ILU(0) of the local Schur complement
        // C - F B^-1 E on C's pattern, and the global interface system is
        // S = S~ + C_o (C_o: couplings to other blocks' interface rows).
        //   forward  z = L^-1 r                       (x_L = M_B f, g - F x_L)
        //   x_S = U_S^-1 z_S, then schur_iters times
        //        x_S <- U_S^-1 (z_S - L_S^-1 C_o x_S)  (block-Jacobi on S)
        //   x_B = U_B^-1 (z_B - E~ x_S)              (x_L = M_B (f - E y))
        // With schur_iters = 0 this is the block-Jacobi apply in the
        // interface-last order.
        std::vector<double> zf(N), x(N), xn(N), xg(N);
#pragma omp parallel for schedule(dynamic)
        for (int b = 0; b < nb; ++b) {
            const int r0 = bstart[b], r1 = bstart[b + 1], i0 = fifc[b];
            for (int q = r0; q < r1; ++q) {
                double acc = r[frow[q]];
                for (int p = fptr[q]; p < fdiag[q]; ++p) acc -= LU[p] * zf[fcol[p]];
                zf[q] = acc;
            }
            for (int q = r1 - 1; q >= i0; --q) {
                double acc = zf[q];
                for (int p = fdiag[q] + 1; p < fptr[q + 1]; ++p) acc -= LU[p] * x[fcol[p]];
                x[q] = acc * LU[fdiag[q]];
            }
        }
        for (int it = 0; it < schur_iters; ++it) {
            for (int q = 0; q < N; ++q) xg[frow[q]] = x[q];
#pragma omp parallel for schedule(dynamic)
            for (int b = 0; b < nb; ++b) {
                const int r1 = bstart[b + 1], i0 = fifc[b];
                // c = L_S^-1 C_o x_S (interior entries of L meet zeros)
                for (int q = i0; q < r1; ++q) {
                    double acc = 0.0;
                    for (int p = optr[q]; p < optr[q + 1]; ++p) acc += J[osrc[p]] * xg[ocol[p]];
                    for (int p = fptr[q]; p < fdiag[q]; ++p)
                        if (fcol[p] >= i0) acc -= LU[p] * xn[fcol[p]];
                    xn[q] = acc;
                }
                for (int q = i0; q < r1; ++q) xn[q] = zf[q] - xn[q];
                for (int q = r1 - 1; q >= i0; --q) {
                    double acc = xn[q];
                    for (int p = fdiag[q] + 1; p < fptr[q + 1]; ++p) acc -= LU[p] * xn[fcol[p]];
                    xn[q] = acc * LU[fdiag[q]];
                }
            }
            for (int b = 0; b < nb; ++b)
                for (int q = fifc[b]; q < bstart[b + 1]; ++q) x[q] = xn[q];
        }
#pragma omp parallel for schedule(dynamic)
        for (int b = 0; b < nb; ++b) {
            const int r0 = bstart[b], i0 = fifc[b];
            for (int q = i0 - 1; q >= r0; --q) {
                double acc = zf[q];
                for (int p = fdiag[q] + 1; p < fptr[q + 1]; ++p) acc -= LU[p] * x[fcol[p]];
                x[q] = acc * LU[fdiag[q]];
            }
            for (int q = r0; q < bstart[b + 1]; ++q) z[frow[q]] = x[q];
        }
        return;
    }
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < nb; ++b) {
        const int r0 = bstart[b], r1 = bstart[b + 1];
        std::vector<double> x(r1 - r0);
        for (int q = r0; q < r1; ++q) {
            double acc = r[frow[q]];
            for (int p = fptr[q]; p < fdiag[q]; ++p) acc -= LU[p] * x[fcol[p] - r0];
            x[q - r0] = acc;
        }
        for (int q = r1 - 1; q >= r0; --q) {
            double acc = x[q - r0];
            for (int p = fdiag[q] + 1; p < fptr[q + 1]; ++p) acc -= LU[p] * x[fcol[p] - r0];
            x[q - r0] = acc * LU[fdiag[q]];
        }
        for (int q = r0; q < r1; ++q) z[frow[q]] = x[q - r0];
    }
}

// restarted GMRES with modified Gram-Schmidt (decomp/gmres.c:412-511), left
// preconditioned and scaled by the error weights as IDAS SPGMR runs it
// inside Newton: minimises ||D P^-1 (b - J x)||, zero initial guess
int Oracle::gmres(double cj, const double* y, const double* yp, const double* F0,
                  const double* ewt, const double* b, double* x, int m, int max_restarts,
                  double tol, int* iters, double* rn, long* njv, long* nps) {
    const double sqrtN = std::sqrt((double)N);
    std::vector<std::vector<double>> V(m + 1, std::vector<double>(N));
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), w(N), z(N), t(N), Jz(N);
    std::fill(x, x + N, 0.0);
    auto wrms_of = [&](const std::vector<double>& v) {
        double s = 0.0;
        for (int i = 0; i < N; ++i) { double q = v[i] * ewt[i]; s += q * q; }
        return std::sqrt(s / N);
    };
    const double g0 = omp_get_wtime();
    double t_jv = 0.0, t_ps = 0.0;
    auto jtimes = [&](const std::vector<double>& v, std::vector<double>& out) {
        const double a = omp_get_wtime();
        double nv = wrms_of(v);
        double sigma = nv > 0 ? 1.0 / nv : 1.0;
        jv(0.0, cj, y, yp, F0, v.data(), sigma, out.data());
        (*njv)++;
        t_jv += omp_get_wtime() - a;
    };
    auto precond = [&](const double* r, double* z) {
        const double a = omp_get_wtime();
        psolve(r, z);
        t_ps += omp_get_wtime() - a;
    };
    struct Book {   // books the time split when the solve returns
        Oracle* o; const double& g0; double& t_jv; double& t_ps; long* njv; long* nps; long njv0, nps0; int* its;
        ~Book() {
            const double all = omp_get_wtime() - g0;
            o->tm[1] += t_jv; o->tm[4] += t_ps; o->tm[5] += all - t_jv - t_ps;
            o->cnt[1] += *njv - njv0; o->cnt[3] += *nps - nps0; o->cnt[4] += *its;
        }
    } book{this, g0, t_jv, t_ps, njv, nps, *njv, *nps, iters};
    *iters = 0;
    int total = 0;
    double rnorm = 0.0;
    bool have_x = false;
    std::vector<double> xv(N, 0.0);
    for (int cycle = 0; cycle <= max_restarts; ++cycle) {
        if (have_x) jtimes(xv, Jz);
        for (int i = 0; i < N; ++i) t[i] = have_x ? b[i] - Jz[i] : b[i];
        precond(t.data(), z.data());
        (*nps)++;
        double beta = 0.0;
        for (int i = 0; i < N; ++i) {
            V[0][i] = ewt[i] * z[i];
            beta += V[0][i] * V[0][i];
        }
        beta = std::sqrt(beta);
        rnorm = beta / sqrtN;
        if (!std::isfinite(beta)) { *iters = total; *rn = rnorm; return 2; }
        if (rnorm <= tol) break;
        for (int i = 0; i < N; ++i) V[0][i] /= beta;
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        bool conv = false;
        for (; j < m; ++j) {
            for (int i = 0; i < N; ++i) t[i] = V[j][i] / ewt[i];
            jtimes(t, Jz);
            precond(Jz.data(), z.data());
            (*nps)++;
            for (int i = 0; i < N; ++i) w[i] = ewt[i] * z[i];
            std::vector<double> hcol(j + 2);
            for (int l = 0; l <= j; ++l) {   // modified Gram-Schmidt (gmres.c:412-511)
                double s = 0.0;
                for (int i = 0; i < N; ++i) s += V[l][i] * w[i];
                hcol[l] = s;
                for (int i = 0; i < N; ++i) w[i] -= s * V[l][i];
            }
            double hn = 0.0;
            for (int i = 0; i < N; ++i) hn += w[i] * w[i];
            hn = std::sqrt(hn);
            hcol[j + 1] = hn;
            ++total;
            if (hn > 0) for (int i = 0; i < N; ++i) V[j + 1][i] = w[i] / hn;
            for (int l = 0; l < j; ++l) {
                double t0 = cs[l] * hcol[l] + sn[l] * hcol[l + 1];
                double t1 = -sn[l] * hcol[l] + cs[l] * hcol[l + 1];
                hcol[l] = t0;
                hcol[l + 1] = t1;
            }
            double den = std::hypot(hcol[j], hcol[j + 1]);
            cs[j] = den == 0.0 ? 1.0 : hcol[j] / den;
            sn[j] = den == 0.0 ? 0.0 : hcol[j + 1] / den;
            hcol[j] = den;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            for (int l = 0; l <= j; ++l) H[(size_t)l * m + j] = hcol[l];
            rnorm = std::fabs(g[j + 1]) / sqrtN;
            if (rnorm <= tol || hn == 0.0) { ++j; conv = true; break; }
        }
        std::vector<double> yv(j);
        for (int i = j - 1; i >= 0; --i) {
            double s = g[i];
            for (int l = i + 1; l < j; ++l) s -= H[(size_t)i * m + l] * yv[l];
            yv[i] = H[(size_t)i * m + i] != 0.0 ? s / H[(size_t)i * m + i] : 0.0;
        }
        std::fill(t.begin(), t.end(), 0.0);
        for (int l = 0; l < j; ++l)
            for (int i = 0; i < N; ++i) t[i] += yv[l] * V[l][i];
        for (int i = 0; i < N; ++i) xv[i] += t[i] / ewt[i];
        have_x = true;
        if (conv) {
            std::copy(xv.begin(), xv.end(), x);
            *iters = total;
            *rn = rnorm;
            return 0;
        }
    }
    std::copy(xv.begin(), xv.end(), x);
    *iters = total;
    *rn = rnorm;
    return rnorm <= tol ? 0 : 1;
}

// ---------------------------------------------------------------- integrator
struct CpuOps {
    Oracle& o;
    const fvm_opts& opt;
    int N, nblocks;
    std::vector<double> phi[7], y, yp, e, ewt, F, x;
    double tcur = 0.0;
    CpuOps(Oracle& oo, const fvm_opts& op, int nb) : o(oo), opt(op), N(oo.N), nblocks(nb) {
        for (auto& p : phi) p.assign(N, 0.0);
        y.assign(N, 0.0); yp.assign(N, 0.0); e.assign(N, 0.0); ewt.assign(N, 1.0);
        F.assign(N, 0.0); x.assign(N, 0.0);
    }
    double wrms(const std::vector<double>& v) const {
        double s = 0.0;
        for (int i = 0; i < N; ++i) { double q = v[i] * ewt[i]; s += q * q; }
        return std::sqrt(s / N);
    }
    void set_time(double t) { tcur = t; }
    void ewt_from_phi0(double rtol, double atol) {
        for (int i = 0; i < N; ++i) ewt[i] = 1.0 / (rtol * std::fabs(phi[0][i]) + atol);
    }
    void begin_step() {
        const double a = omp_get_wtime();
        o.begin_step(tcur, phi[0].data(), yp.data());
        o.tm[0] += omp_get_wtime() - a;
        o.cnt[0]++;
    }
    void phi_scale(int j0, int j1, const double* f) {
        for (int j = j0; j <= j1; ++j)
            for (int i = 0; i < N; ++i) phi[j][i] *= f[j];
    }
    void predict(int k, const double* gamma, double) {
        for (int i = 0; i < N; ++i) {
            double s = phi[0][i], sp = 0.0;
            for (int j = 1; j <= k; ++j) { s += phi[j][i]; sp += gamma[j] * phi[j][i]; }
            y[i] = s; yp[i] = sp; e[i] = 0.0;
        }
        pn = wrms(y);
    }
    double pn = 0.0;
    double pred_norm() const { return pn; }
    void set_order(int) {}
    void residual() {
        const double a = omp_get_wtime();
        o.residual(tcur, y.data(), yp.data(), F.data());
        o.tm[0] += omp_get_wtime() - a;
        o.cnt[0]++;
    }
    int psetup(double cj, double h) { return o.timed_psetup(tcur, cj, h, y.data(), yp.data(), F.data(), ewt.data(), nblocks); }
    int gmres(double cj, double tol, int* its, double* rn, long* nps, long* njv) {
        return o.gmres(cj, y.data(), yp.data(), F.data(), ewt.data(), F.data(), x.data(), opt.krylov_dim,
                       opt.max_restarts, tol, its, rn, njv, nps);
    }
    double newton_update(double cj) {
        for (int i = 0; i < N; ++i) { y[i] -= x[i]; yp[i] -= cj * x[i]; e[i] -= x[i]; }
        return wrms(x);
    }
    void err_norms(int k, double out[4]) {
        std::vector<double> d(N);
        out[0] = wrms(e);
        for (int i = 0; i < N; ++i) d[i] = phi[k][i] + e[i];
        out[1] = wrms(d);
        if (k >= 2) { for (int i = 0; i < N; ++i) d[i] = phi[k - 1][i] + phi[k][i] + e[i]; out[2] = wrms(d); }
        else out[2] = 0.0;
        if (k + 1 < 7) { for (int i = 0; i < N; ++i) d[i] = e[i] - phi[k + 1][i]; out[3] = wrms(d); }
        else out[3] = 0.0;
    }
    void phi_update(int k, int set_kp2) {
        for (int i = 0; i < N; ++i) {
            if (set_kp2) phi[k + 1][i] = e[i];
            phi[k][i] += e[i];
            for (int j = k - 1; j >= 0; --j) phi[j][i] += phi[j + 1][i];
        }
    }
    bool newton_guess(double, double, double) { return false; }
};

} // namespace orc

using namespace orc;

extern "C" {

typedef struct orc_ctx orc_ctx;

orc_ctx* orc_create(const fvm_mesh* m, const fvm_physics* ph, char* err, int errlen) {
    try {
        Oracle* o = new Oracle();
        o->build(m, ph);
        return reinterpret_cast<orc_ctx*>(o);
    } catch (const std::exception& ex) {
        if (err && errlen > 0) { std::strncpy(err, ex.what(), errlen - 1); err[errlen - 1] = 0; }
        return nullptr;
    }
}

void orc_destroy(orc_ctx* c) { delete reinterpret_cast<Oracle*>(c); }

int orc_sizes(orc_ctx* c, int* E, int* Fi, int* Fall, int* ncolours) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    if (E) *E = o->E;
    if (Fi) *Fi = o->Fi;
    if (Fall) *Fall = o->Fall;
    if (ncolours) *ncolours = o->ncol;
    return 0;
}

int orc_volumes(orc_ctx* c, double* V) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    std::copy(o->cvvol.begin(), o->cvvol.end(), V);
    return 0;
}

// per-node sum of area-weighted CV-face normals (outward from the CV):
// zero for interior nodes of a closed mesh
int orc_cv_normal_sums(orc_ctx* c, double* S) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    std::fill(S, S + 3 * (size_t)o->N, 0.0);
    for (int f = 0; f < o->Fi; ++f) {
        P3 n = o->cf_normal[f];
        int b = o->cf_back[f], fr = o->cf_front[f];
        S[3 * b] += n.x; S[3 * b + 1] += n.y; S[3 * b + 2] += n.z;
        S[3 * fr] -= n.x; S[3 * fr + 1] -= n.y; S[3 * fr + 2] -= n.z;
    }
    return 0;
}

int orc_residual(orc_ctx* c, double t, const double* y, const double* yp, double* res) {
    reinterpret_cast<Oracle*>(c)->residual(t, y, yp, res);
    return 0;
}

int orc_begin_step(orc_ctx* c, double t, const double* y, const double* yp) {
    reinterpret_cast<Oracle*>(c)->begin_step(t, y, yp);
    return 0;
}

// upwind weights per edge: 1 = front upwind, 0 = back, 2 = averaged
int orc_upwind(orc_ctx* c, int* w) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    for (int g = 0; g < o->E; ++g) w[g] = o->w_front[g] == 1.0 ? 1 : (o->w_back[g] == 1.0 ? 0 : 2);
    return 0;
}

int orc_edges(orc_ctx* c, int* front, int* back) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    std::copy(o->edge_front.begin(), o->edge_front.end(), front);
    std::copy(o->edge_back.begin(), o->edge_back.end(), back);
    return 0;
}

int orc_ahh(orc_ctx* c, double* a) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    std::copy(o->ahh.begin(), o->ahh.end(), a);
    return 0;
}

int orc_jv(orc_ctx* c, double t, double cj, const double* y, const double* yp, const double* F0,
           const double* v, double sigma, double* Jv) {
    reinterpret_cast<Oracle*>(c)->jv(t, cj, y, yp, F0, v, sigma, Jv);
    return 0;
}

int orc_psetup(orc_ctx* c, double t, double cj, double h, const double* y, const double* yp,
               const double* F0, const double* ewt, int nblocks) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    o->psetup(t, cj, h, y, yp, F0, ewt, nblocks);
    return o->ilu_factor();
}

int orc_jacobian_nnz(orc_ctx* c) { return (int)reinterpret_cast<Oracle*>(c)->jcol.size(); }

int orc_jacobian(orc_ctx* c, int* rowptr, int* col, double* val, int* colour) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    if (rowptr) std::copy(o->jrow.begin(), o->jrow.end(), rowptr);
    if (col) std::copy(o->jcol.begin(), o->jcol.end(), col);
    if (val) std::copy(o->J.begin(), o->J.end(), val);
    if (colour) std::copy(o->colour.begin(), o->colour.end(), colour);
    return 0;
}

// factor a given Jacobian (values over the oracle's pattern) with nblocks
// contiguous row blocks, so that preconditioner applies can be compared on
// identical matrices
int orc_factor_given(orc_ctx* c, const double* val, int nblocks) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    if (!o->pat_built) return -1;
    std::copy(val, val + o->J.size(), o->J.begin());
    int nb = std::max(1, nblocks);
    o->bstart.resize(nb + 1);
    for (int b = 0; b <= nb; ++b) o->bstart[b] = (int)(((long)o->N * b) / nb);
    return o->ilu_factor();
}

// van Genuchten Sw, dSw/dh, krw for one zone (saturation, CPU branch)
int orc_vg(double alpha, double n, double S_r, int count, const double* h, double* Sw, double* dSw,
           double* krw) {
    Zone z{0, 0, 0, 0.5, alpha, n, 1.0 - 1.0 / n, S_r};
    std::vector<double> hh(h, h + count), a, b, k;
    saturation(hh, z, a, b, k);
    std::copy(a.begin(), a.end(), Sw);
    std::copy(b.begin(), b.end(), dSw);
    std::copy(k.begin(), k.end(), krw);
    return 0;
}

// Schur interface coupling of the block ILU(0) (< 0 off, >= 0 interface
// iterations per apply); takes effect at the next factorisation
int orc_set_schur(orc_ctx* c, int iters) {
    reinterpret_cast<Oracle*>(c)->schur_iters = iters;
    return 0;
}

// interface rows of each block after the last factorisation (0 when the
// Schur coupling is off)
int orc_schur_interface_rows(orc_ctx* c) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    if (o->schur_iters < 0) return 0;
    long n = 0;
    for (size_t b = 0; b + 1 < o->bstart.size(); ++b) n += o->bstart[b + 1] - o->fifc[b];
    return (int)n;
}

int orc_psolve(orc_ctx* c, const double* r, double* z) {
    reinterpret_cast<Oracle*>(c)->psolve(r, z);
    return 0;
}

int orc_gmres(orc_ctx* c, double cj, const double* y, const double* yp, const double* F0,
              const double* ewt, const double* b, double* x, int m, int max_restarts, double tol,
              int* iters, double* rn) {
    long njv = 0, nps = 0;
    return reinterpret_cast<Oracle*>(c)->gmres(cj, y, yp, F0, ewt, b, x, m, max_restarts, tol, iters, rn, &njv, &nps);
}

// The time loop of fvm_integrate (t_end a stop time) and, with n_out > 0,
// of fvm_integrate_outputs: steps with no stop time, each output time's head
// y_out[i N ..] and derivative yp_out[i N ..] interpolated from the step that
// reached it (IDAIntegrator::advance(next_time), ida_integrator.h:325-340).
static int orc_run(orc_ctx* c, const fvm_opts* opts, int nblocks, double t0, double t_end,
                   const double* y0, double* y_end, fvm_stats* stats, int n_out, const double* t_out,
                   double* y_out, double* yp_out) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    const int N = o->N;
    const double wall0 = omp_get_wtime();
    CpuOps ops(*o, *opts, nblocks);
    fvmb::BdfOptions bo;
    bo.rtol = opts->rtol;
    bo.atol = opts->atol;
    bo.max_order = opts->max_order;
    bo.hmax = opts->hmax;
    if (opts->eps_lin > 0.0) bo.eps_lin = opts->eps_lin;
    if (opts->cj_refresh > 1.0) bo.cj_refresh = opts->cj_refresh;
    if (opts->psetup_age > 0) bo.psetup_age = opts->psetup_age;
    fvmb::BdfController<CpuOps> ctl(ops, bo);
    long nre0 = o->n_res;
    std::fill(o->w_front.begin(), o->w_front.end(), 0.5);   // averaged weights before step 1
    std::fill(o->w_back.begin(), o->w_back.end(), 0.5);
    // y'0 = F(t0, y0, 0) / ahh on free rows (fvmpor_ODE_impl.cpp:45-57)
    std::vector<double> zero(N, 0.0), F(N);
    o->residual(t0, y0, zero.data(), F.data());
    std::vector<double> yp0(N, 0.0);
    for (int i = 0; i < N; ++i)
        if (!o->is_dirichlet[i] && o->ahh[i] != 0.0) yp0[i] = F[i] / o->ahh[i];
    for (int i = 0; i < N; ++i) ops.ewt[i] = 1.0 / (opts->rtol * std::fabs(y0[i]) + opts->atol);
    double h0 = fvmb::bdf_first_step(t0, t_end, ops.wrms(yp0), opts->h0, opts->hmax);
    for (int i = 0; i < N; ++i) { ops.phi[0][i] = y0[i]; ops.phi[1][i] = h0 * yp0[i]; ops.yp[i] = yp0[i]; }
    ctl.start(t0, h0);
    int rc = 0, done = 0;
    const double tstop = n_out > 0 ? std::numeric_limits<double>::infinity() : t_end;
    while (n_out > 0 ? done < n_out : ctl.t < t_end) {
        if (opts->max_steps > 0 && ctl.st.nst >= opts->max_steps) { rc = 1; break; }
        rc = ctl.step(tstop);
        if (rc != 0) break;
        if (n_out > 0) {
            for (; done < n_out && t_out[done] <= ctl.t; ++done) {
                double cf[7], df[7];
                const int k = ctl.interp_coefs(t_out[done], cf, df);
                double* yo = y_out + (size_t)done * N;
                double* ypo = yp_out ? yp_out + (size_t)done * N : nullptr;
                for (int i = 0; i < N; ++i) {
                    double s = ops.phi[0][i], sp = 0.0;
                    for (int j = 1; j <= k; ++j) { s += cf[j] * ops.phi[j][i]; sp += df[j] * ops.phi[j][i]; }
                    yo[i] = s;
                    if (ypo) ypo[i] = sp;
                }
            }
        } else if (t_end - ctl.t <= 1e-12 * std::max(1.0, std::fabs(t_end))) {
            ctl.t = t_end;
        }
    }
    if (y_end) std::copy(ops.phi[0].begin(), ops.phi[0].end(), y_end);
    o->last_trace.swap(ctl.trace);
    o->cnt[5] += ctl.st.nni;
    o->cnt[6] += ctl.st.nst;
    o->tm[6] += omp_get_wtime() - wall0;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->nst = ctl.st.nst; stats->nre = o->n_res - nre0; stats->nni = ctl.st.nni;
        stats->nli = ctl.st.nli; stats->npe = ctl.st.npe; stats->nps = ctl.st.nps;
        stats->ncfn = ctl.st.ncfn; stats->ncfl = ctl.st.ncfl; stats->netf = ctl.st.netf;
        stats->last_order = ctl.st.last_order; stats->last_h = ctl.st.last_h; stats->t = ctl.t;
    }
    return rc;
}

int orc_integrate(orc_ctx* c, const fvm_opts* opts, int nblocks, double t0, double t_end,
                  const double* y0, double* y_end, fvm_stats* stats) {
    return orc_run(c, opts, nblocks, t0, t_end, y0, y_end, stats, 0, nullptr, nullptr, nullptr);
}

// the dense-output coefficients of the controller, for a known-answer test
int orc_interp_coefs(const double* psi, int k, double delt, double* c, double* d) {
    if (k < 1 || k > 6) return -1;
    fvmb::bdf_interp_coefs(psi, k, delt, 7, c, d);
    return 0;
}

// fvm_integrate_outputs restated; the output times are ascending and after t0
int orc_integrate_outputs(orc_ctx* c, const fvm_opts* opts, int nblocks, double t0, const double* y0,
                          int n_out, const double* t_out, double* y_out, double* yp_out, fvm_stats* stats) {
    if (n_out < 1) return -1;
    for (int i = 0; i < n_out; ++i)
        if (!std::isfinite(t_out[i]) || !(t_out[i] > (i ? t_out[i - 1] : t0))) return -1;
    return orc_run(c, opts, nblocks, t0, t_out[n_out - 1], y0, nullptr, stats, n_out, t_out, y_out, yp_out);
}

int orc_threads(void) { return omp_get_max_threads(); }

// The same replay driven by the product's controller template
// (fvmb::bdf_replay_step: modified divided differences) with the oracle's
// kernels.  Against orc_replay this compares the controller's predictor and
// corrector formulas with the independent Lagrange-form restatement, on
// identical kernels.
int orc_replay_controller(orc_ctx* c, const fvm_opts* opts, int nblocks, double t0, const double* y0, double h0,
                          long n, const fvm_step_record* steps, double newton_tol, int max_newton, double* y_end,
                          fvm_stats* stats) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    if (!opts || !y0 || !steps || n < 1 || !(h0 > 0) || !(newton_tol > 0) || max_newton < 1) return -1;
    const int N = o->N;
    CpuOps ops(*o, *opts, nblocks);
    fvmb::BdfOptions bo;
    bo.rtol = opts->rtol;
    bo.atol = opts->atol;
    bo.max_order = opts->max_order;
    fvmb::BdfController<CpuOps> ctl(ops, bo);
    std::fill(o->w_front.begin(), o->w_front.end(), 0.5);
    std::fill(o->w_back.begin(), o->w_back.end(), 0.5);
    std::vector<double> zero(N, 0.0), F(N), yp0(N, 0.0);
    o->residual(t0, y0, zero.data(), F.data());
    for (int i = 0; i < N; ++i)
        if (!o->is_dirichlet[i] && o->ahh[i] != 0.0) yp0[i] = F[i] / o->ahh[i];
    for (int i = 0; i < N; ++i) { ops.phi[0][i] = y0[i]; ops.phi[1][i] = h0 * yp0[i]; ops.yp[i] = yp0[i]; }
    ctl.start(t0, h0);
    int rc = 0;
    for (long s = 0; s < n; ++s) {
        const int r = fvmb::bdf_replay_step(ctl, steps[s].h, steps[s].order, newton_tol, max_newton);
        if (r < 0) return r;
        if (r == 1) rc = 1;
    }
    if (y_end) std::copy(ops.phi[0].begin(), ops.phi[0].end(), y_end);
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->nst = ctl.st.nst; stats->nni = ctl.st.nni; stats->nli = ctl.st.nli; stats->npe = ctl.st.npe;
        stats->nps = ctl.st.nps; stats->t = ctl.t;
    }
    return rc;
}

// initial head: the Dirichlet value on Dirichlet rows, water_table minus the
// elevation elsewhere (set_initial_conditions, examples/fvmporMinlin/vs.h:8-32)
int orc_initial_head(orc_ctx* c, double water_table, double* y) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    for (int i = 0; i < o->N; ++i) y[i] = water_table - (o->dim == 2 ? o->X[i].y : o->X[i].z);
    for (size_t d = 0; d < o->dirichlet_nodes.size(); ++d) y[o->dirichlet_nodes[d]] = o->h_dirichlet[d];
    return 0;
}

// copies up to cap records of the last adaptive integration; returns the count
long orc_step_trace(orc_ctx* c, fvm_step_record* out, long cap) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    const long n = (long)o->last_trace.size();
    if (out && cap > 0) std::copy(o->last_trace.begin(), o->last_trace.begin() + std::min(n, cap), out);
    return n;
}

// time split and work counters since creation or the last reset (reset != 0
// zeroes them after reading); either pointer may be NULL
int orc_timers(orc_ctx* c, double* tm, long* cnt, int reset) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    if (tm) std::copy(o->tm, o->tm + 7, tm);
    if (cnt) std::copy(o->cnt, o->cnt + 7, cnt);
    if (reset) {
        std::fill(o->tm, o->tm + 7, 0.0);
        std::fill(o->cnt, o->cnt + 7, 0L);
    }
    return 0;
}

// Replay of a given sequence of accepted BDF steps (step sizes and orders),
// with each corrector solved to a tight tolerance.
//
// This is an independent restatement of the fixed-leading-coefficient BDF
// step of DASSL / IDA (Brenan, Campbell & Petzold 1996, ch. 5; Hindmarsh et
// al., ACM TOMS 31(3), 2005) that the reference's IDAIntegrator drives
// (include/fvm/integrators/ida_integrator.h:296-321).  It does not use the
// modified divided differences of the adaptive controller: the predictor of
// a step of order k is the polynomial through the k + 1 newest solution
// values, evaluated in Lagrange form,
//   y_pred = sum_i l_i(t) Y_i,   y'_pred = sum_i l_i'(t) Y_i,
// and the corrector solves G(y) = F(t, y, y'_pred + cj (y - y_pred)) = 0 with
// cj = (1 + 1/2 + ... + 1/k) / h.  Before the first step the history holds
// y0 and the point (t0 - h0, y0 - h0 y'0), the line through y0 with slope
// y'0 that the divided-difference form starts from (phi_1 = h0 y'0).
// y'0 = F(t0, y0, 0) / ahh on free rows (fvmpor_ODE_impl.cpp:34-58).  The
// upwind directions are frozen at the start of every step from the newest
// solution (fvmpor_ODE_impl.cpp:118-141).  Newton: one preconditioner set-up
// at the predictor, then updates until ||delta||_wrms <= newton_tol (error
// weights 1/(rtol |y_n| + atol)), GMRES solved to 0.05 newton_tol.  Returns 0
// on success, 1 if some step's Newton iteration did not reach newton_tol
// within max_newton updates (the state is still advanced), < 0 on bad input.
int orc_replay(orc_ctx* c, const fvm_opts* opts, int nblocks, double t0, const double* y0, double h0, long n,
               const fvm_step_record* steps, double newton_tol, int max_newton, double* y_end, fvm_stats* stats) {
    Oracle* o = reinterpret_cast<Oracle*>(c);
    if (!opts || !y0 || !steps || n < 1 || !(h0 > 0) || !(newton_tol > 0) || max_newton < 1) return -1;
    const int N = o->N;
    const double wall0 = omp_get_wtime();
    std::fill(o->w_front.begin(), o->w_front.end(), 0.5);
    std::fill(o->w_back.begin(), o->w_back.end(), 0.5);
    std::vector<double> zero(N, 0.0), F(N), yp(N, 0.0), y(N), x(N), ewt(N);
    o->residual(t0, y0, zero.data(), F.data());
    for (int i = 0; i < N; ++i)
        if (!o->is_dirichlet[i] && o->ahh[i] != 0.0) yp[i] = F[i] / o->ahh[i];
    // history, newest first: (time, solution)
    std::vector<double> Th;
    std::vector<std::vector<double>> Yh;
    Th.push_back(t0);
    Yh.emplace_back(y0, y0 + N);
    Th.push_back(t0 - h0);
    Yh.emplace_back(N);
    for (int i = 0; i < N; ++i) Yh[1][i] = y0[i] - h0 * yp[i];
    double t = t0;
    long nni = 0, nli = 0, npe = 0, nps = 0, nre0 = o->n_res;
    int rc = 0;
    for (long s = 0; s < n; ++s) {
        const double h = steps[s].h;
        const int k = steps[s].order;
        if (!(h > 0) || k < 1 || k > 5 || (size_t)k + 1 > Th.size()) return -2;
        const double tn = t + h;
        // Lagrange weights over the k + 1 newest nodes and their derivatives
        double l[6], dl[6];
        for (int i = 0; i <= k; ++i) {
            double prod = 1.0, dsum = 0.0;
            for (int j = 0; j <= k; ++j) {
                if (j == i) continue;
                prod *= (tn - Th[j]) / (Th[i] - Th[j]);
            }
            for (int m = 0; m <= k; ++m) {
                if (m == i) continue;
                double term = 1.0 / (Th[i] - Th[m]);
                for (int j = 0; j <= k; ++j)
                    if (j != i && j != m) term *= (tn - Th[j]) / (Th[i] - Th[j]);
                dsum += term;
            }
            l[i] = prod;
            dl[i] = dsum;
        }
        const std::vector<double>& yn = Yh[0];
        for (int i = 0; i < N; ++i) ewt[i] = 1.0 / (opts->rtol * std::fabs(yn[i]) + opts->atol);
        {
            const double a = omp_get_wtime();
            o->begin_step(t, yn.data(), yp.data());
            o->tm[0] += omp_get_wtime() - a;
            o->cnt[0]++;
        }
        double alphas = 0.0;
        for (int j = 1; j <= k; ++j) alphas += 1.0 / j;
        const double cj = alphas / h;
        std::vector<double> ypred(N), yppred(N);
        for (int i = 0; i < N; ++i) {
            double s0 = 0.0, s1 = 0.0;
            for (int q = 0; q <= k; ++q) { s0 += l[q] * Yh[q][i]; s1 += dl[q] * Yh[q][i]; }
            ypred[i] = s0;
            yppred[i] = s1;
        }
        y = ypred;
        yp = yppred;
        bool conv = false;
        for (int m = 0; m < max_newton; ++m) {
            {
                const double a = omp_get_wtime();
                o->residual(tn, y.data(), yp.data(), F.data());
                o->tm[0] += omp_get_wtime() - a;
                o->cnt[0]++;
            }
            if (m == 0) {
                if (o->timed_psetup(tn, cj, h, y.data(), yp.data(), F.data(), ewt.data(), nblocks)) return -3;
                npe++;
            }
            int its = 0;
            double rn = 0.0;
            long njv = 0, np = 0;
            o->gmres(cj, y.data(), yp.data(), F.data(), ewt.data(), F.data(), x.data(), opts->krylov_dim,
                     opts->max_restarts, 0.05 * newton_tol, &its, &rn, &njv, &np);
            nli += its;
            nps += np;
            nni++;
            double d2 = 0.0;
            for (int i = 0; i < N; ++i) {
                y[i] -= x[i];
                yp[i] -= cj * x[i];
                const double q = x[i] * ewt[i];
                d2 += q * q;
            }
            if (std::sqrt(d2 / N) <= newton_tol) { conv = true; break; }
        }
        if (!conv) rc = 1;
        Th.insert(Th.begin(), tn);
        Yh.insert(Yh.begin(), y);
        if (Th.size() > 7) { Th.pop_back(); Yh.pop_back(); }
        t = tn;
    }
    if (y_end) std::copy(Yh[0].begin(), Yh[0].end(), y_end);
    o->cnt[5] += nni;
    o->cnt[6] += n;
    o->tm[6] += omp_get_wtime() - wall0;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->nst = n; stats->nre = o->n_res - nre0; stats->nni = nni; stats->nli = nli; stats->npe = npe;
        stats->nps = nps; stats->last_order = steps[n - 1].order; stats->last_h = steps[n - 1].h; stats->t = t;
    }
    return rc;
}

}  // extern "C"
