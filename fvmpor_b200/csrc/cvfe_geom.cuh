// CVFE element geometry shared by the host set-up and the device kernels.
//
// Vertex-centred control volumes are the median-dual cells of the simplex
// mesh.  For every element edge (a, b) the reference builds one CV face:
//   2D: the segment from the edge midpoint to the element centroid
//       (src/fvm/mesh.cpp:941-1010),
//   3D: the quadrilateral (edge midpoint, face centroid, element centroid,
//       face centroid) (src/fvm/mesh.cpp:844-939),
// with its area-weighted normal pointing from one edge node to the other
// (include/fvm/impl/mesh/cvface_inline.h:110-118, 164-175), and evaluates
// the head gradient there from the linear shape functions
// (examples/fvmporMinlin/shape.cpp:27-60 triangle, :98-135 tetrahedron).
// For linear simplices these reduce to closed forms: the face area vector
// of edge (a, b) with opposite nodes c (, d) is
//   2D: S = R90((2 x_c - x_a - x_b) / 6)
//   3D: S = (x_c + x_d - x_a - x_b) x (x_d - x_c) / 24
// oriented so that S . (x_b - x_a) > 0, the gradients are constant over the
// element, and every sub-control volume holds |element| / (dim + 1).
//
// Local edge tables follow Mesh::construct_edges_and_faces
// (src/fvm/mesh.cpp:383-441): triangle 0-1 1-2 2-0; tetrahedron
// 0-1 1-2 2-0 0-3 1-3 2-3.
#pragma once

#ifdef __CUDACC__
#define FVM_HD __host__ __device__ __forceinline__
#else
#define FVM_HD inline
#endif

namespace fvmb {

FVM_HD int tri_edge_a(int f) { return f; }
FVM_HD int tri_edge_b(int f) { return f == 2 ? 0 : f + 1; }
FVM_HD int tri_edge_c(int f) { return f == 0 ? 2 : f - 1; }
FVM_HD int tet_edge_a(int f) { return f < 3 ? f : f - 3; }
FVM_HD int tet_edge_b(int f) { return f < 3 ? (f == 2 ? 0 : f + 1) : 3; }
FVM_HD int tet_edge_c(int f) { return f == 0 ? 2 : (f == 1 ? 0 : (f == 2 ? 1 : (f == 3 ? 1 : 0))); }
FVM_HD int tet_edge_d(int f) { return f < 3 ? 3 : (f == 5 ? 1 : 2); }

// Per-element flux coefficients: for face f,
//   qdotn_f / krw = sum_k C[f][k] h_k + G[f]
// with C[f][k] = -sum_d K_d S_fd dN_k/dx_d and G[f] = -K_v S_fv (v the
// vertical axis: y in 2D, z in 3D), i.e. S_f . q for q = -K (grad h + e_v)
// (process_fluxes, examples/fvmporMinlin/fvmpor.h:692-711, K stored
// negated at :632-643).  Also returns the face areas |S_f| and the element
// measure (area / volume, positive).  Returns false for a degenerate
// element.
FVM_HD bool tet_coefficients(const double* x0, const double* x1, const double* x2,
                             const double* x3, double Kx, double Ky, double Kz,
                             double C[6][4], double G[6], double area[6], double* vol) {
    const double* X[4] = {x0, x1, x2, x3};
    double u[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
    double v[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
    double w[3] = {x3[0] - x0[0], x3[1] - x0[1], x3[2] - x0[2]};
    // rows of the inverse Jacobian: grad N1 = (v x w)/det etc.
    double vw[3] = {v[1] * w[2] - v[2] * w[1], v[2] * w[0] - v[0] * w[2], v[0] * w[1] - v[1] * w[0]};
    double wu[3] = {w[1] * u[2] - w[2] * u[1], w[2] * u[0] - w[0] * u[2], w[0] * u[1] - w[1] * u[0]};
    double uv[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    double det = u[0] * vw[0] + u[1] * vw[1] + u[2] * vw[2];
    if (!(det != 0.0)) return false;
    double id = 1.0 / det;
    double g[4][3];
    for (int d = 0; d < 3; ++d) {
        g[1][d] = vw[d] * id;
        g[2][d] = wu[d] * id;
        g[3][d] = uv[d] * id;
        g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
    }
    *vol = (det > 0 ? det : -det) / 6.0;
    const double K[3] = {Kx, Ky, Kz};
    for (int f = 0; f < 6; ++f) {
        const double* xa = X[tet_edge_a(f)];
        const double* xb = X[tet_edge_b(f)];
        const double* xc = X[tet_edge_c(f)];
        const double* xd = X[tet_edge_d(f)];
        double p[3], q[3], e[3];
        for (int d = 0; d < 3; ++d) {
            p[d] = (xc[d] + xd[d]) - (xa[d] + xb[d]);
            q[d] = xd[d] - xc[d];
            e[d] = xb[d] - xa[d];
        }
        double S[3] = {(p[1] * q[2] - p[2] * q[1]) * (1.0 / 24.0),
                       (p[2] * q[0] - p[0] * q[2]) * (1.0 / 24.0),
                       (p[0] * q[1] - p[1] * q[0]) * (1.0 / 24.0)};
        if (S[0] * e[0] + S[1] * e[1] + S[2] * e[2] < 0.0) { S[0] = -S[0]; S[1] = -S[1]; S[2] = -S[2]; }
        double KS[3] = {K[0] * S[0], K[1] * S[1], K[2] * S[2]};
        for (int k = 0; k < 4; ++k) C[f][k] = -(KS[0] * g[k][0] + KS[1] * g[k][1] + KS[2] * g[k][2]);
        G[f] = -KS[2];
        double a2 = S[0] * S[0] + S[1] * S[1] + S[2] * S[2];
        area[f] = sqrt(a2);
    }
    return true;
}

// The six face fluxes S_f . (-K (grad h + e_z)) of one tetrahedron straight
// from its vertices, for the element pass that rebuilds the geometry
// instead of streaming stored coefficients.  With node 0 at the origin
// (u, v, w = x1, x2, x3 - x0) the shape-function gradients are the
// cofactor rows v x w, w x u, u x v over det = u . (v x w), so
//   grad h = G / det,  G = (h1 - h0) v x w + (h2 - h0) w x u + (h3 - h0) u x v.
// The raw face vector P_f = (x_c + x_d - x_a - x_b) x (x_d - x_c) obeys
// P_f . (x_b - x_a) = 2 det(x_b - x_a, x_c - x_a, x_d - x_a) = 2 s_f det,
// s_f the parity of the vertex permutation (a, b, c, d) of face f (odd only
// for face 4 of the edge table), so the oriented area vector of the
// closed form above is S_f = s_f sign(det) P_f / 24 and
//   q_f = s_f P_f . t,   t = -K (G / |det| + sign(det) e_z) / 24.
// Same quantity as sum_k C[f][k] h_k + G[f] of tet_coefficients, with the
// head gradient formed once per element instead of once per face.
FVM_HD void tet_face_fluxes(const double* x0, const double* x1, const double* x2, const double* x3,
                            double Kx, double Ky, double Kz, double h0, double h1, double h2,
                            double h3, double q[6]) {
    const double u[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
    const double v[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
    const double w[3] = {x3[0] - x0[0], x3[1] - x0[1], x3[2] - x0[2]};
    const double vw[3] = {v[1] * w[2] - v[2] * w[1], v[2] * w[0] - v[0] * w[2], v[0] * w[1] - v[1] * w[0]};
    const double wu[3] = {w[1] * u[2] - w[2] * u[1], w[2] * u[0] - w[0] * u[2], w[0] * u[1] - w[1] * u[0]};
    const double uv[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    const double det = u[0] * vw[0] + u[1] * vw[1] + u[2] * vw[2];
    const double d1 = h1 - h0, d2 = h2 - h0, d3 = h3 - h0;
    const double r = 1.0 / (det > 0.0 ? det : -det);
    const double sg = det > 0.0 ? 1.0 : -1.0;
    const double c24 = 1.0 / 24.0;
    double t[3];
    t[0] = -(Kx * ((d1 * vw[0] + d2 * wu[0] + d3 * uv[0]) * r)) * c24;
    t[1] = -(Ky * ((d1 * vw[1] + d2 * wu[1] + d3 * uv[1]) * r)) * c24;
    t[2] = -(Kz * ((d1 * vw[2] + d2 * wu[2] + d3 * uv[2]) * r + sg)) * c24;
    // q_f = s_f (p x r') . t = s_f p . (r' x t)
    auto face = [&](const double p0, const double p1, const double p2, const double* rr) {
        double a0 = rr[1] * t[2] - rr[2] * t[1];
        double a1 = rr[2] * t[0] - rr[0] * t[2];
        double a2 = rr[0] * t[1] - rr[1] * t[0];
        return p0 * a0 + p1 * a1 + p2 * a2;
    };
    double rr[3];
    // f0: a0 b1 c2 d3   p = v + w - u, r' = w - v
    rr[0] = w[0] - v[0]; rr[1] = w[1] - v[1]; rr[2] = w[2] - v[2];
    q[0] = face(v[0] + w[0] - u[0], v[1] + w[1] - u[1], v[2] + w[2] - u[2], rr);
    // f1: a1 b2 c0 d3   p = w - u - v, r' = w
    q[1] = face(w[0] - u[0] - v[0], w[1] - u[1] - v[1], w[2] - u[2] - v[2], w);
    // f2: a2 b0 c1 d3   p = u + w - v, r' = w - u
    rr[0] = w[0] - u[0]; rr[1] = w[1] - u[1]; rr[2] = w[2] - u[2];
    q[2] = face(u[0] + w[0] - v[0], u[1] + w[1] - v[1], u[2] + w[2] - v[2], rr);
    // f3: a0 b3 c1 d2   p = u + v - w, r' = v - u
    rr[0] = v[0] - u[0]; rr[1] = v[1] - u[1]; rr[2] = v[2] - u[2];
    q[3] = face(u[0] + v[0] - w[0], u[1] + v[1] - w[1], u[2] + v[2] - w[2], rr);
    // f4: a1 b3 c0 d2   p = v - u - w, r' = v   (odd permutation)
    q[4] = -face(v[0] - u[0] - w[0], v[1] - u[1] - w[1], v[2] - u[2] - w[2], v);
    // f5: a2 b3 c0 d1   p = u - v - w, r' = u
    q[5] = face(u[0] - v[0] - w[0], u[1] - v[1] - w[1], u[2] - v[2] - w[2], u);
}

// The coefficients C[f][k], G[f] of tet_coefficients rebuilt from the
// vertices with the relations of tet_face_fluxes: S_f = s_f sign(det) P_f /
// 24 and grad N_k = cof_k / det (cof_1..3 = v x w, w x u, u x v, cof_0 =
// -(cof_1 + cof_2 + cof_3)), so
//   C[f][k] = -s_f (K o P_f) . cof_k / (24 |det|),
//   G[f]    = -s_f sign(det) K_z P_fz / 24.
// No square roots and no orientation tests; for kernels that need the
// coefficients themselves (the finite-difference Jacobian).
FVM_HD void tet_coefficients_fast(const double* x0, const double* x1, const double* x2, const double* x3,
                                  double Kx, double Ky, double Kz, double C[6][4], double G[6]) {
    const double u[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
    const double v[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
    const double w[3] = {x3[0] - x0[0], x3[1] - x0[1], x3[2] - x0[2]};
    double cof[4][3];
    cof[1][0] = v[1] * w[2] - v[2] * w[1]; cof[1][1] = v[2] * w[0] - v[0] * w[2]; cof[1][2] = v[0] * w[1] - v[1] * w[0];
    cof[2][0] = w[1] * u[2] - w[2] * u[1]; cof[2][1] = w[2] * u[0] - w[0] * u[2]; cof[2][2] = w[0] * u[1] - w[1] * u[0];
    cof[3][0] = u[1] * v[2] - u[2] * v[1]; cof[3][1] = u[2] * v[0] - u[0] * v[2]; cof[3][2] = u[0] * v[1] - u[1] * v[0];
    for (int d = 0; d < 3; ++d) cof[0][d] = -(cof[1][d] + cof[2][d] + cof[3][d]);
    const double det = u[0] * cof[1][0] + u[1] * cof[1][1] + u[2] * cof[1][2];
    const double r24 = 1.0 / (24.0 * (det > 0.0 ? det : -det));
    const double sg24 = (det > 0.0 ? 1.0 : -1.0) / 24.0;
    // p = x_c + x_d - x_a - x_b, r' = x_d - x_c per face (node 0 at the origin)
    double p[6][3], rr[6][3];
    for (int d = 0; d < 3; ++d) {
        p[0][d] = v[d] + w[d] - u[d]; rr[0][d] = w[d] - v[d];
        p[1][d] = w[d] - u[d] - v[d]; rr[1][d] = w[d];
        p[2][d] = u[d] + w[d] - v[d]; rr[2][d] = w[d] - u[d];
        p[3][d] = u[d] + v[d] - w[d]; rr[3][d] = v[d] - u[d];
        p[4][d] = v[d] - u[d] - w[d]; rr[4][d] = v[d];
        p[5][d] = u[d] - v[d] - w[d]; rr[5][d] = u[d];
    }
    for (int f = 0; f < 6; ++f) {
        const double sf = f == 4 ? -1.0 : 1.0;
        double P0 = p[f][1] * rr[f][2] - p[f][2] * rr[f][1];
        double P1 = p[f][2] * rr[f][0] - p[f][0] * rr[f][2];
        double P2 = p[f][0] * rr[f][1] - p[f][1] * rr[f][0];
        const double KP0 = Kx * P0, KP1 = Ky * P1, KP2 = Kz * P2;
        for (int k = 0; k < 4; ++k)
            C[f][k] = -sf * ((KP0 * cof[k][0] + KP1 * cof[k][1] + KP2 * cof[k][2]) * r24);
        G[f] = -sf * (KP2 * sg24);
    }
}

FVM_HD bool tri_coefficients(const double* x0, const double* x1, const double* x2, double Kx,
                             double Ky, double C[3][3], double G[3], double area[3],
                             double* vol) {
    const double* X[3] = {x0, x1, x2};
    double det = (x1[0] - x0[0]) * (x2[1] - x0[1]) - (x1[1] - x0[1]) * (x2[0] - x0[0]);
    if (!(det != 0.0)) return false;
    double id = 1.0 / det;
    double g[3][2] = {{(x1[1] - x2[1]) * id, (x2[0] - x1[0]) * id},
                      {(x2[1] - x0[1]) * id, (x0[0] - x2[0]) * id},
                      {(x0[1] - x1[1]) * id, (x1[0] - x0[0]) * id}};
    *vol = (det > 0 ? det : -det) * 0.5;
    for (int f = 0; f < 3; ++f) {
        const double* xa = X[tri_edge_a(f)];
        const double* xb = X[tri_edge_b(f)];
        const double* xc = X[tri_edge_c(f)];
        double s0 = (2.0 * xc[0] - xa[0] - xb[0]) * (1.0 / 6.0);
        double s1 = (2.0 * xc[1] - xa[1] - xb[1]) * (1.0 / 6.0);
        double S[2] = {s1, -s0};
        if (S[0] * (xb[0] - xa[0]) + S[1] * (xb[1] - xa[1]) < 0.0) { S[0] = -S[0]; S[1] = -S[1]; }
        double KS[2] = {Kx * S[0], Ky * S[1]};
        for (int k = 0; k < 3; ++k) C[f][k] = -(KS[0] * g[k][0] + KS[1] * g[k][1]);
        G[f] = -KS[1];
        area[f] = sqrt(S[0] * S[0] + S[1] * S[1]);
    }
    return true;
}

} // namespace fvmb
