// .pmesh mesh files and VTK XML output.
//
// Reader: the text format Mesh::read_mesh_data parses (src/fvm/mesh.cpp:
// 102-366): a header (domain count and id, the vtxdist array, node and
// element counts), external node ids, one line per node (x y z, the number
// of boundary tags, the tags) and one line per element (gmsh type,
// physical tag + 100, node ids, one boundary id per local face).  The hot
// path covers triangles (type 2) and tetrahedra (type 4) of a single
// domain; other element types and meshes with halo nodes are rejected with
// an error.  Local faces follow construct_edges_and_faces (mesh.cpp:368-
// 480): triangle faces (0,1) (1,2) (2,0); tetrahedron faces (0,1,2)
// (0,1,3) (0,2,3) (1,2,3).  A tagged face that several elements share is
// kept once, for the first element, as the reference's face set does.
//
// Node ordering: with FVM_PMESH_RCM the nodes are renumbered by reverse
// Cuthill-McKee as Mesh::reorder_nodes_edges does (mesh.cpp:116-148 calls
// find_RCM_from_edges, :1571-1613, which hands the edge graph to Boost
// Graph's cuthill_mckee_ordering; Boost is not in the tree).  The method
// restated here is the one that routine publishes (George & Liu, "Computer
// Solution of Large Sparse Positive Definite Systems", 1981, ch. 4): for
// each connected component, in order of its lowest node id, a
// pseudo-peripheral start node from repeated level-structure sweeps (the
// lowest-degree node of the last level, first in sweep order on ties,
// until the eccentricity stops growing); then a breadth-first sweep that
// enqueues each node's unvisited neighbours, taken in ascending id order,
// sorted stably by ascending degree; the whole sequence reversed.
//
// Writer: the UnstructuredGrid piece and the PUnstructuredGrid header that
// util::Solution::write_timestep_VTK_XML / write_timestep_header_VTK_XML
// produce (include/util/solution.h:175-357), with the same file names
// (<stem>_dom<rank>_<step>.vtu, <stem>_head_<step>.pvtu) and arrays
// (pressure_head, dom, Points, connectivity, offsets, types), so existing
// ParaView state files keep working.  Values are rounded to Float32, the
// declared type, and written with 9 significant digits (exact) instead of
// the stream default of 6.
#include "common.hpp"

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>

namespace fvmb {

namespace {

template <class T>
T* copy_vec(const std::vector<T>& v) {
    T* p = (T*)std::malloc(std::max<size_t>(1, v.size()) * sizeof(T));
    if (!p) throw Error("out of host memory", -1);
    if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

// whitespace-separated tokens with the line number for error messages
struct Tokens {
    std::ifstream in;
    std::string path;
    long line = 1;
    bool next(std::string& tok) {
        tok.clear();
        int c;
        while ((c = in.get()) != EOF) {
            if (c == '\n') ++line;
            if (!std::isspace(c)) break;
        }
        if (c == EOF) return false;
        tok.push_back((char)c);
        while ((c = in.peek()) != EOF && !std::isspace(c)) tok.push_back((char)in.get());
        return true;
    }
    [[noreturn]] void fail(const std::string& what) {
        throw Error(path + ":" + std::to_string(line) + ": " + what, -2);
    }
    long integer(const char* what) {
        std::string t;
        if (!next(t)) fail(std::string("unexpected end of file reading ") + what);
        char* end = nullptr;
        errno = 0;
        long v = std::strtol(t.c_str(), &end, 10);
        if (errno || *end) fail(std::string("expected an integer for ") + what + ", got '" + t + "'");
        return v;
    }
    double real(const char* what) {
        std::string t;
        if (!next(t)) fail(std::string("unexpected end of file reading ") + what);
        char* end = nullptr;
        errno = 0;
        double v = std::strtod(t.c_str(), &end);
        if (errno == ERANGE || *end) fail(std::string("expected a number for ") + what + ", got '" + t + "'");
        return v;
    }
};

const int kTriFace[3][2] = {{0, 1}, {1, 2}, {2, 0}};
const int kTetFace[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

struct Graph {
    std::vector<int> ptr, adj;  // neighbours in ascending id order
};

Graph node_graph(int n, int npe, const std::vector<int>& en) {
    std::vector<std::pair<int, int>> e;
    size_t ne = en.size() / npe;
    e.reserve(ne * npe * (npe - 1));
    for (size_t k = 0; k < ne; ++k)
        for (int a = 0; a < npe; ++a)
            for (int b = 0; b < npe; ++b)
                if (a != b) e.emplace_back(en[k * npe + a], en[k * npe + b]);
    std::sort(e.begin(), e.end());
    e.erase(std::unique(e.begin(), e.end()), e.end());
    Graph g;
    g.ptr.assign(n + 1, 0);
    for (auto& p : e) g.ptr[p.first + 1]++;
    for (int i = 0; i < n; ++i) g.ptr[i + 1] += g.ptr[i];
    g.adj.resize(e.size());
    for (size_t i = 0; i < e.size(); ++i) g.adj[i] = e[i].second;
    return g;
}

int bandwidth(const Graph& g, const std::vector<int>& pos) {
    int bw = 0;
    for (int u = 0; u + 1 < (int)g.ptr.size(); ++u)
        for (int k = g.ptr[u]; k < g.ptr[u + 1]; ++k) bw = std::max(bw, std::abs(pos[u] - pos[g.adj[k]]));
    return bw;
}

// level-structure sweep from r: returns the lowest-degree node of the last
// level (first in sweep order on ties) and its eccentricity
int last_level_min(const Graph& g, int r, int& ecc, std::vector<int>& mark, int stamp, std::vector<int>& q) {
    q.clear();
    q.push_back(r);
    mark[r] = stamp;
    size_t lo = 0;
    ecc = -1;
    int w = r;
    while (lo < q.size()) {
        size_t hi = q.size();
        ++ecc;
        w = q[lo];
        for (size_t i = lo; i < hi; ++i) {
            int u = q[i];
            if (g.ptr[u + 1] - g.ptr[u] < g.ptr[w + 1] - g.ptr[w]) w = u;
            for (int k = g.ptr[u]; k < g.ptr[u + 1]; ++k) {
                int v = g.adj[k];
                if (mark[v] != stamp) { mark[v] = stamp; q.push_back(v); }
            }
        }
        lo = hi;
    }
    return w;
}

// new -> old node order
std::vector<int> rcm_order(const Graph& g, int n) {
    std::vector<int> comp_of(n, -1), reps, q;
    for (int v = 0; v < n; ++v) {
        if (comp_of[v] >= 0) continue;
        int c = (int)reps.size();
        reps.push_back(v);
        q.assign(1, v);
        comp_of[v] = c;
        for (size_t i = 0; i < q.size(); ++i)
            for (int k = g.ptr[q[i]]; k < g.ptr[q[i] + 1]; ++k)
                if (comp_of[g.adj[k]] < 0) { comp_of[g.adj[k]] = c; q.push_back(g.adj[k]); }
    }
    std::vector<int> mark(n, 0);
    int stamp = 0;
    std::vector<int> order;
    order.reserve(n);
    std::vector<char> seen(n, 0);
    auto deg = [&](int u) { return g.ptr[u + 1] - g.ptr[u]; };
    for (int r : reps) {
        int er, ex;
        int x = last_level_min(g, r, er, mark, ++stamp, q);
        int y = last_level_min(g, x, ex, mark, ++stamp, q);
        while (ex > er) {
            r = x; er = ex; x = y;
            y = last_level_min(g, x, ex, mark, ++stamp, q);
        }
        size_t head = order.size();
        order.push_back(x);
        seen[x] = 1;
        while (head < order.size()) {
            int u = order[head++];
            size_t first = order.size();
            for (int k = g.ptr[u]; k < g.ptr[u + 1]; ++k) {
                int v = g.adj[k];
                if (!seen[v]) { seen[v] = 1; order.push_back(v); }
            }
            std::stable_sort(order.begin() + first, order.end(), [&](int a, int b) { return deg(a) < deg(b); });
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

void read_pmesh(const char* path, int flags, fvm_pmesh* out) {
    Tokens t;
    t.path = path ? path : "";
    t.in.open(t.path);
    if (!t.in) throw Error("cannot open " + t.path, -1);
    int n_dom = (int)t.integer("the domain count");
    int dom_id = (int)t.integer("the domain id");
    if (n_dom < 1 || dom_id < 0 || dom_id >= n_dom) t.fail("bad domain header");
    for (int i = 0; i <= n_dom; ++i) t.integer("vtxdist");
    long n_gbl = t.integer("the global node count");
    long n_int = t.integer("the interior node count");
    long n_bnd = t.integer("the boundary node count");
    long n_ext = t.integer("the external node count");
    long ne_int = t.integer("the interior element count");
    long ne_bnd = t.integer("the boundary element count");
    (void)n_gbl;
    if (n_int < 0 || n_bnd < 0 || n_ext < 0 || ne_int < 0 || ne_bnd < 0) t.fail("negative count");
    if (n_ext != 0)
        throw Error(t.path + ": " + std::to_string(n_ext) +
                        " external (halo) nodes: multi-domain meshes are outside the single-GPU hot path",
                    -3);
    long n = n_int + n_bnd, ne = ne_int + ne_bnd;
    if (n < 1 || ne < 1 || n > (1L << 30) || ne > (1L << 30)) t.fail("node or element count out of range");

    std::vector<double> xyz(3 * n);
    std::vector<int> bc_ptr(n + 1, 0), bc;
    for (long i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) xyz[3 * i + d] = t.real("a node coordinate");
        long nbc = t.integer("a node's boundary-tag count");
        if (nbc < 0 || nbc > 64) t.fail("bad boundary-tag count");
        for (long k = 0; k < nbc; ++k) bc.push_back((int)t.integer("a node boundary tag"));
        bc_ptr[i + 1] = (int)bc.size();
    }
    int dim = 0, npe = 0, nfe = 0;
    std::vector<int> en, etag, bn, be, bt;
    std::set<std::vector<int>> tagged;
    for (long k = 0; k < ne; ++k) {
        int type = (int)t.integer("an element type");
        int tag = (int)t.integer("an element physical tag") - 100;
        int d = type == 2 ? 2 : type == 4 ? 3 : 0;
        if (!d)
            throw Error(t.path + ":" + std::to_string(t.line) + ": element type " + std::to_string(type) +
                            " (" + (type == 3 ? "quadrilateral" : type == 5 ? "hexahedron" : type == 6 ? "prism" : "unknown") +
                            "): the CVFE hot path covers triangles (2) and tetrahedra (4)",
                        -4);
        if (dim && d != dim) t.fail("triangles and tetrahedra mixed in one mesh");
        dim = d; npe = d + 1; nfe = d + 1;
        int ids[4];
        for (int a = 0; a < npe; ++a) {
            long v = t.integer("an element node id");
            if (v < 0 || v >= n) t.fail("element node id " + std::to_string(v) + " out of range");
            ids[a] = (int)v;
            en.push_back((int)v);
        }
        for (int a = 0; a < npe; ++a)
            for (int b = a + 1; b < npe; ++b)
                if (ids[a] == ids[b]) t.fail("repeated node in an element");
        etag.push_back(tag);
        for (int f = 0; f < nfe; ++f) {
            int id = (int)t.integer("a face boundary id");
            if (id < 0) t.fail("negative face boundary id");
            if (id == 0) continue;
            std::vector<int> fn;
            if (d == 2) fn = {ids[kTriFace[f][0]], ids[kTriFace[f][1]]};
            else fn = {ids[kTetFace[f][0]], ids[kTetFace[f][1]], ids[kTetFace[f][2]]};
            std::vector<int> key = fn;
            std::sort(key.begin(), key.end());
            if (!tagged.insert(key).second) continue;
            bn.insert(bn.end(), fn.begin(), fn.end());
            be.push_back((int)k);
            bt.push_back(id);
        }
    }

    Graph g = node_graph((int)n, npe, en);
    std::vector<int> ident(n);
    for (long i = 0; i < n; ++i) ident[i] = (int)i;
    int bw0 = bandwidth(g, ident);
    std::vector<int> perm = ident;  // new -> file
    if (flags & FVM_PMESH_RCM) perm = rcm_order(g, (int)n);
    std::vector<int> q(n);          // file -> new
    for (long i = 0; i < n; ++i) q[perm[i]] = (int)i;
    int bw1 = bandwidth(g, q);

    std::vector<double> xyz2(3 * n);
    std::vector<int> ptr2(n + 1, 0), bc2;
    for (long i = 0; i < n; ++i) {
        int o = perm[i];
        for (int d2 = 0; d2 < 3; ++d2) xyz2[3 * i + d2] = xyz[3 * o + d2];
        bc2.insert(bc2.end(), bc.begin() + bc_ptr[o], bc.begin() + bc_ptr[o + 1]);
        ptr2[i + 1] = (int)bc2.size();
    }
    for (auto& v : en) v = q[v];
    for (auto& v : bn) v = q[v];

    std::memset(out, 0, sizeof(*out));
    out->n_dom = n_dom;
    out->dom_id = dom_id;
    out->dim = dim;
    out->n_nodes = (int)n;
    out->n_elements = (int)ne;
    out->n_bfaces = (int)bt.size();
    out->coords = copy_vec(xyz2);
    out->elem_nodes = copy_vec(en);
    out->elem_tag = copy_vec(etag);
    out->bface_nodes = copy_vec(bn);
    out->bface_elem = copy_vec(be);
    out->bface_tag = copy_vec(bt);
    out->node_bc_ptr = copy_vec(ptr2);
    out->node_bc = copy_vec(bc2);
    out->perm = copy_vec(perm);
    out->bandwidth_file = bw0;
    out->bandwidth = bw1;
}

void write_pmesh(const char* path, const fvm_pmesh* m) {
    if (!m || (m->dim != 2 && m->dim != 3) || m->n_nodes < 1 || m->n_elements < 1)
        throw Error("fvm_pmesh_write: bad mesh", -1);
    const int npe = m->dim + 1, nfe = m->dim + 1, nfn = m->dim;
    // element-local face boundary ids
    std::vector<int> fid((size_t)m->n_elements * nfe, 0);
    for (int b = 0; b < m->n_bfaces; ++b) {
        int k = m->bface_elem[b];
        if (k < 0 || k >= m->n_elements) throw Error("fvm_pmesh_write: bface_elem out of range", -1);
        std::vector<int> key(m->bface_nodes + (size_t)b * nfn, m->bface_nodes + (size_t)(b + 1) * nfn);
        std::sort(key.begin(), key.end());
        int found = -1;
        for (int f = 0; f < nfe && found < 0; ++f) {
            std::vector<int> fk;
            for (int a = 0; a < nfn; ++a)
                fk.push_back(m->elem_nodes[(size_t)k * npe + (m->dim == 2 ? kTriFace[f][a] : kTetFace[f][a])]);
            std::sort(fk.begin(), fk.end());
            if (fk == key) found = f;
        }
        if (found < 0) throw Error("fvm_pmesh_write: boundary face " + std::to_string(b) + " is not a face of its element", -1);
        fid[(size_t)k * nfe + found] = m->bface_tag[b];
    }
    FILE* f = std::fopen(path, "w");
    if (!f) throw Error(std::string("cannot write ") + path, -1);
    std::fprintf(f, "1 0\n0 %d \n%d %d 0 0 %d 0\n", m->n_nodes, m->n_nodes, m->n_nodes, m->n_elements);
    for (int i = 0; i < m->n_nodes; ++i) {
        const double* x = m->coords + 3 * (size_t)i;
        int a = m->node_bc_ptr ? m->node_bc_ptr[i] : 0, b = m->node_bc_ptr ? m->node_bc_ptr[i + 1] : 0;
        std::fprintf(f, "%.17g %.17g %.17g %d", x[0], x[1], x[2], b - a);
        for (int k = a; k < b; ++k) std::fprintf(f, " %d", m->node_bc[k]);
        std::fputc('\n', f);
    }
    for (int k = 0; k < m->n_elements; ++k) {
        std::fprintf(f, "%d %d    ", m->dim == 2 ? 2 : 4, m->elem_tag[k] + 100);
        for (int a = 0; a < npe; ++a) std::fprintf(f, " %d", m->elem_nodes[(size_t)k * npe + a]);
        std::fputs("     ", f);
        for (int a = 0; a < nfe; ++a) std::fprintf(f, " %d", fid[(size_t)k * nfe + a]);
        std::fputc('\n', f);
    }
    if (std::fclose(f) != 0) throw Error(std::string("error writing ") + path, -1);
}

void write_vtu(const char* stem, int step, int rank, int n_ranks, const fvm_mesh* m, const double* head) {
    if (!stem || !m || !head || step < 0 || rank < 0 || n_ranks < 1 || rank >= n_ranks)
        throw Error("fvm_write_vtu: bad arguments", -1);
    const int npe = m->dim + 1;
    const int vtk_type = m->dim == 2 ? 5 : 10;  // VTK_TRIANGLE, VTK_TETRA
    std::string s(stem);
    std::string piece = s + "_dom" + std::to_string(rank) + "_" + std::to_string(step) + ".vtu";
    FILE* f = std::fopen(piece.c_str(), "w");
    if (!f) throw Error("cannot write " + piece, -1);
    std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\">\n  <UnstructuredGrid>\n");
    std::fprintf(f, "    <Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n", m->n_nodes, m->n_elements);
    std::fprintf(f, "      <PointData Scalars=\"pressure_head\">\n");
    std::fprintf(f, "        <DataArray Name=\"pressure_head\" type=\"Float32\" format=\"ascii\">\n          ");
    // values rounded to Float32 first, then written with the 9 digits that
    // reproduce a Float32 exactly
    auto f32 = [](double v) { return (double)(float)v; };
    for (int i = 0; i < m->n_nodes; ++i) std::fprintf(f, "%.9g ", f32(head[i]));
    std::fprintf(f, "\n        </DataArray>\n      </PointData>\n");
    std::fprintf(f, "      <CellData Scalars=\"dom\">\n        <DataArray Name=\"dom\" type=\"Int32\" format=\"ascii\">\n");
    for (int k = 0; k < m->n_elements; ++k) std::fprintf(f, "%d ", rank);
    std::fprintf(f, "\n        </DataArray>\n      </CellData>\n");
    std::fprintf(f, "      <Points>\n        <DataArray NumberOfComponents=\"3\" type=\"Float32\" format=\"ascii\">\n          ");
    for (int i = 0; i < m->n_nodes; ++i)
        std::fprintf(f, "%.9g %.9g %.9g ", f32(m->coords[3 * (size_t)i]), f32(m->coords[3 * (size_t)i + 1]),
                     f32(m->coords[3 * (size_t)i + 2]));
    std::fprintf(f, "\n        </DataArray>\n      </Points>\n      <Cells>\n");
    std::fprintf(f, "        <DataArray Name=\"connectivity\" type=\"Int32\" format=\"ascii\">\n          ");
    for (int k = 0; k < m->n_elements; ++k) {
        for (int a = 0; a < npe; ++a) std::fprintf(f, "%d ", m->elem_nodes[(size_t)k * npe + a]);
        std::fputc(' ', f);
    }
    std::fprintf(f, "\n        </DataArray>\n        <DataArray Name=\"offsets\" type=\"Int32\" format=\"ascii\">\n          ");
    for (int k = 0; k < m->n_elements; ++k) std::fprintf(f, "%lld ", (long long)(k + 1) * npe);
    std::fprintf(f, "\n        </DataArray>\n        <DataArray Name=\"types\" type=\"UInt8\" format=\"ascii\">\n          ");
    for (int k = 0; k < m->n_elements; ++k) std::fprintf(f, "%d ", vtk_type);
    std::fprintf(f, "\n        </DataArray>\n      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n");
    if (std::fclose(f) != 0) throw Error("error writing " + piece, -1);
    if (rank != 0) return;
    std::string head_name = s + "_head_" + std::to_string(step) + ".pvtu";
    f = std::fopen(head_name.c_str(), "w");
    if (!f) throw Error("cannot write " + head_name, -1);
    std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"PUnstructuredGrid\">\n  <PUnstructuredGrid GhostLevel=\"0\">\n");
    std::fprintf(f, "    <PPointData Scalars=\"pressure_head\">\n      <PDataArray Name=\"pressure_head\" type=\"Float32\" format=\"ascii\"/>\n    </PPointData>\n");
    std::fprintf(f, "    <PCellData Scalars=\"dom\">\n      <PDataArray Name=\"dom\" type=\"Int32\" format=\"ascii\"/>\n    </PCellData>\n");
    std::fprintf(f, "    <PPoints>\n      <PDataArray NumberOfComponents=\"3\" type=\"Float32\" format=\"ascii\"/>\n    </PPoints>\n");
    std::fprintf(f, "    <PCells>\n      <PDataArray Name=\"connectivity\" type=\"Int32\" format=\"ascii\"/>\n");
    std::fprintf(f, "      <PDataArray Name=\"offsets\" type=\"Int32\" format=\"ascii\"/>\n");
    std::fprintf(f, "      <PDataArray Name=\"types\" type=\"UInt8\" format=\"ascii\"/>\n    </PCells>\n");
    // piece sources are relative to the header's own directory
    std::string base = s.substr(s.find_last_of('/') == std::string::npos ? 0 : s.find_last_of('/') + 1);
    for (int r = 0; r < n_ranks; ++r)
        std::fprintf(f, "    <Piece Source=\"%s_dom%d_%d.vtu\"/>\n", base.c_str(), r, step);
    std::fprintf(f, "  </PUnstructuredGrid>\n</VTKFile>\n");
    if (std::fclose(f) != 0) throw Error("error writing " + head_name, -1);
}

}  // namespace

}  // namespace fvmb

using namespace fvmb;

extern "C" int fvm_pmesh_read(const char* path, int flags, fvm_pmesh* out) {
    if (!out) return -1;
    try {
        read_pmesh(path, flags, out);
        return 0;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_pmesh_write(const char* path, const fvm_pmesh* m) {
    try {
        write_pmesh(path, m);
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" void fvm_pmesh_free(fvm_pmesh* m) {
    if (!m) return;
    std::free(m->coords); std::free(m->elem_nodes); std::free(m->elem_tag);
    std::free(m->bface_nodes); std::free(m->bface_elem); std::free(m->bface_tag);
    std::free(m->node_bc_ptr); std::free(m->node_bc); std::free(m->perm);
    std::memset(m, 0, sizeof(*m));
}

extern "C" int fvm_problem_from_pmesh(const fvm_pmesh* m, int n_zones, const fvm_zone* zones, int n_bcs,
                                      const fvm_bc* bcs, double rho0, fvm_problem* out) {
    try {
        if (!m || !out || !zones || n_zones < 1 || (n_bcs > 0 && !bcs) || n_bcs < 0)
            throw Error("fvm_problem_from_pmesh: bad arguments", -1);
        const int npe = m->dim + 1;
        std::map<int, int> bc_type;
        for (int i = 0; i < n_bcs; ++i) bc_type[bcs[i].tag] = bcs[i].type;
        std::vector<int> nt(m->n_nodes, 0);
        for (int i = 0; i < m->n_nodes; ++i)
            for (int k = m->node_bc_ptr[i]; k < m->node_bc_ptr[i + 1]; ++k) {
                auto it = bc_type.find(m->node_bc[k]);
                if (it != bc_type.end() && (it->second == 1 || it->second == 4)) nt[i] = m->node_bc[k];
            }
        for (int k = 0; k < m->n_elements; ++k)
            if (m->elem_tag[k] < 0 || m->elem_tag[k] >= n_zones)
                throw Error("fvm_problem_from_pmesh: element " + std::to_string(k) + " has physical tag " +
                                std::to_string(m->elem_tag[k] + 100) + ", outside the " + std::to_string(n_zones) +
                                " zones given",
                            -1);
        for (int b = 0; b < m->n_bfaces; ++b)
            if (!bc_type.count(m->bface_tag[b]))
                throw Error("fvm_problem_from_pmesh: boundary tag " + std::to_string(m->bface_tag[b]) +
                                " has no boundary condition",
                            -1);
        std::memset(out, 0, sizeof(*out));
        auto dup = [](const void* src, size_t bytes) {
            void* p = std::malloc(std::max<size_t>(1, bytes));
            if (!p) throw Error("out of host memory", -1);
            if (bytes) std::memcpy(p, src, bytes);
            return p;
        };
        out->coords = (double*)dup(m->coords, sizeof(double) * 3 * m->n_nodes);
        out->elem_nodes = (int*)dup(m->elem_nodes, sizeof(int) * (size_t)npe * m->n_elements);
        out->elem_zone = (int*)dup(m->elem_tag, sizeof(int) * m->n_elements);
        out->elem_K = nullptr;
        out->bface_nodes = (int*)dup(m->bface_nodes, sizeof(int) * (size_t)m->dim * m->n_bfaces);
        out->bface_elem = (int*)dup(m->bface_elem, sizeof(int) * m->n_bfaces);
        out->bface_tag = (int*)dup(m->bface_tag, sizeof(int) * m->n_bfaces);
        out->node_tag = (int*)dup(nt.data(), sizeof(int) * m->n_nodes);
        out->zones = (fvm_zone*)dup(zones, sizeof(fvm_zone) * n_zones);
        out->bcs = (fvm_bc*)dup(bcs, sizeof(fvm_bc) * n_bcs);
        out->grid_dims = (int*)std::calloc(3, sizeof(int));
        if (!out->grid_dims) throw Error("out of host memory", -1);
        fvm_mesh& mm = out->mesh;
        mm.dim = m->dim;
        mm.n_nodes = m->n_nodes;
        mm.n_elements = m->n_elements;
        mm.n_bfaces = m->n_bfaces;
        mm.coords = out->coords; mm.elem_nodes = out->elem_nodes; mm.elem_zone = out->elem_zone;
        mm.elem_K = nullptr; mm.bface_nodes = out->bface_nodes; mm.bface_elem = out->bface_elem;
        mm.bface_tag = out->bface_tag; mm.node_tag = out->node_tag;
        out->phys.n_zones = n_zones;
        out->phys.zones = out->zones;
        out->phys.n_bcs = n_bcs;
        out->phys.bcs = out->bcs;
        out->phys.rho0 = rho0;
        out->water_table = 0.0;
        out->t_end = 0.0;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_write_vtu(const char* stem, int step, int rank, int n_ranks, const fvm_mesh* mesh,
                             const double* head) {
    try {
        write_vtu(stem, step, rank, n_ranks, mesh, head);
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}
