// contact.cuh — candidate predicates and the active-stencil classification
// shared by detection, energy and assembly.
#pragma once
#include "engine.cuh"
#include "physics.cuh"

// ------------------------------------------------------------------ predicates
struct Geo {
    const double* x; const float4* xf; const int2* edges; const int* tris; const int* vbody;
    const int* bscene; const double* planes; const int* sc_plane_begin; const double* mass;
    const double* xbar;
};

// EE candidate test (contact.py:158-168).  Returns the distance used by the
// filter (float32 or float64 closest points) and the clamped parameters.
DV bool ee_test(const Geo& G, int i, int j, int f32, int self_contact, double filt,
                double& s, double& t, double& d) {
    int2 a = G.edges[i], b = G.edges[j];
    if (a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y) return false;
    if (!self_contact && G.vbody[a.x] == G.vbody[b.x]) return false;
    if (f32) {
        float4 pa = G.xf[a.x], qa = G.xf[a.y], pb = G.xf[b.x], qb = G.xf[b.y];
        float p1[3] = {pa.x, pa.y, pa.z}, q1[3] = {qa.x, qa.y, qa.z}, p2[3] = {pb.x, pb.y, pb.z}, q2[3] = {qb.x, qb.y, qb.z};
        float fs, ft, fd;
        seg_seg_f32(p1, q1, p2, q2, 1e-6f, fs, ft, fd);
        s = fs; t = ft; d = fd;
        return fd < __double2float_rn(filt);
    }
    seg_seg_f64(G.x + 3*a.x, G.x + 3*a.y, G.x + 3*b.x, G.x + 3*b.y, 1e-12, s, t, d);
    return d < filt;
}
DV bool pt_test(const Geo& G, int p, int tr, int self_contact, double filt) {
    int a = G.tris[3*tr], b = G.tris[3*tr+1], c = G.tris[3*tr+2];
    if (p == a || p == b || p == c) return false;
    if (!self_contact && G.vbody[p] == G.vbody[a]) return false;
    double f = pt_dist2(G.x + 3*p, G.x + 3*a, G.x + 3*b, G.x + 3*c);
    return f < filt * filt;
}

// Classification of one candidate into an active stencil (abd.py:220-225,
// :351-464).  Returns false if the contact is inactive.  st: vertex ids,
// type T_*, xb: barrier argument.
DV bool classify(const Geo& G, int kind, int a, int b, int f32, double dhat,
                 int4& stv, int& type, double& xb) {
    stv = make_int4(-1, -1, -1, -1);
    if (kind == ABD_CONTACT_EE) {
        int2 ea = G.edges[a], eb = G.edges[b];
        double s, t, d;
        ee_test(G, a, b, f32, 1, 1e300, s, t, d);
        if (!(d < dhat)) return false;
        bool a0 = s == 0.0, a1 = s == 1.0, b0 = t == 0.0, b1 = t == 1.0;
        int i0 = ea.x, i1 = ea.y, i2 = eb.x, i3 = eb.y;
        double f;
        if ((a0 || a1) && (b0 || b1)) {
            type = T_PP;
            stv.x = a0 ? i0 : i1; stv.y = b0 ? i2 : i3;
            f = d2_pp_val(ld3(G.x + 3*stv.x), ld3(G.x + 3*stv.y));
        } else if (a0 || a1 || b0 || b1) {
            type = T_PE;
            if (a0) stv = make_int4(i0, i2, i3, -1);
            else if (a1) stv = make_int4(i1, i2, i3, -1);
            else if (b0) stv = make_int4(i2, i0, i1, -1);
            else stv = make_int4(i3, i0, i1, -1);
            f = d2_pe_val(ld3(G.x + 3*stv.x), ld3(G.x + 3*stv.y), ld3(G.x + 3*stv.z));
        } else {
            type = T_EE;
            stv = make_int4(i0, i1, i2, i3);
            f = d2_ee_line_val(ld3(G.x + 3*i0), ld3(G.x + 3*i1), ld3(G.x + 3*i2), ld3(G.x + 3*i3));
        }
        xb = f32 ? d * d : f;
        return true;
    }
    if (kind == ABD_CONTACT_PT) {
        int t0 = G.tris[3*b], t1 = G.tris[3*b+1], t2 = G.tris[3*b+2];
        int T[3] = {t0, t1, t2};
        int r = pt_region(G.x + 3*a, G.x + 3*t0, G.x + 3*t1, G.x + 3*t2);
        double f;
        d3 P = ld3(G.x + 3*a);
        if (r <= 2) { type = T_PP; stv = make_int4(a, T[r], -1, -1); f = d2_pp_val(P, ld3(G.x + 3*T[r])); }
        else if (r <= 5) {
            type = T_PE; int e0 = T[r-3], e1 = T[(r-3+1)%3];
            stv = make_int4(a, e0, e1, -1);
            f = d2_pe_val(P, ld3(G.x + 3*e0), ld3(G.x + 3*e1));
        } else {
            type = T_PT; stv = make_int4(a, t0, t1, t2);
            f = d2_pt_plane_val(P, ld3(G.x + 3*t0), ld3(G.x + 3*t1), ld3(G.x + 3*t2));
        }
        if (!(f < dhat * dhat)) return false;
        xb = f;
        return true;
    }
    const double* n = G.planes + 4*b;
    double d = n[0] * G.x[3*a] + n[1] * G.x[3*a+1] + n[2] * G.x[3*a+2] - n[3];
    if (!(d < dhat)) return false;
    type = T_PG; stv = make_int4(a, b, -1, -1); xb = d * d;
    return true;
}

