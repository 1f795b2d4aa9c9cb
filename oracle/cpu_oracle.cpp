// CPU oracle for the path-tracing hot path -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of the reference's device code, used by tests/ as
// the checker and by bench.py as the timed CPU baseline.  It is never linked
// into or called by the product library (tfg_b200/libtfgpt.so).
//
// It follows the reference's arithmetic: positions / directions in double
// (Vector3d, vector3d.h:14-143), colours in float (color.h:13-79), the mixed
// float/double intersectors of primitiva.h:121-200, the CWBVH traversal of
// traverse_cwbvh.cuh:51-257 (bfind / prmt / vshl emulated on the host), the
// path loop of render.h:33-466, the RNG of rng.h:12-35 and the small kernels
// of RenderKernel.cu:49-166 and NrcKernel.cu:5-126.  Built with
// -ffp-contract=off so each source operation rounds once.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/tfg_pt.h"

namespace {

// ------------------------------------------------------------------ value types
struct D3 {
    double x, y, z;
    D3() : x(0), y(0), z(0) {}
    D3(double a, double b, double c) : x(a), y(b), z(c) {}
    explicit D3(const TfgVec3d& v) : x(v.x), y(v.y), z(v.z) {}
    D3 operator+(const D3& o) const { return D3(x + o.x, y + o.y, z + o.z); }
    D3 operator-(const D3& o) const { return D3(x - o.x, y - o.y, z - o.z); }
    D3 operator*(double s) const { return D3(x * s, y * s, z * s); }
    D3 operator-() const { return D3(-x, -y, -z); }
    double dot(const D3& o) const { return x * o.x + y * o.y + z * o.z; }
    D3 cross(const D3& o) const { return D3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x); }
    double length() const { return std::sqrt(x * x + y * y + z * z); }
    D3 normalized() const {
        double l = length();
        if (l > 0.0) return *this * (1.0 / l);
        return *this;
    }
    void normalize() {
        double l = length();
        if (l > 0.0) { x /= l; y /= l; z /= l; }
    }
    bool operator!=(const D3& o) const { return !(x == o.x && y == o.y && z == o.z); }
};
inline D3 operator*(double s, const D3& v) { return v * s; }

struct C3 {
    float r, g, b;
    C3() : r(0), g(0), b(0) {}
    C3(float a, float c, float d) : r(a), g(c), b(d) {}
    explicit C3(const TfgColor& c) : r(c.r), g(c.g), b(c.b) {}
    C3 operator+(const C3& o) const { return C3(r + o.r, g + o.g, b + o.b); }
    C3 operator-(const C3& o) const { return C3(r - o.r, g - o.g, b - o.b); }
    C3 operator*(float s) const { return C3(r * s, g * s, b * s); }
    C3 operator*(const C3& o) const { return C3(r * o.r, g * o.g, b * o.b); }
    C3 operator/(float s) const {
        if (s == 0.0f) return C3(0, 0, 0);
        return C3(r / s, g / s, b / s);
    }
    float max() const {
        float m = (r >= g) ? r : g;
        if (b > m) m = b;
        return m;
    }
};

inline TfgColor tc(const C3& c) { return TfgColor{c.r, c.g, c.b}; }
inline TfgVec3d tv(const D3& v) { return TfgVec3d{v.x, v.y, v.z}; }

// ------------------------------------------------------------------ RNG (rng.h:12-35)
inline uint32_t pcg(uint32_t& s) {
    s = s * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
inline float pcgf(uint32_t& s) { return (float)pcg(s) * (1.0f / 4294967296.0f); }
inline uint32_t seed(int px, int py, int frame) {
    uint32_t s = (uint32_t)(py << 16) | (uint32_t)(px & 0xFFFF);
    s ^= (uint32_t)frame * 719393u;
    s = (s ^ 61u) ^ (s >> 16u);
    s *= 0x27d4eb2du;
    s = (s ^ (s >> 15u));
    return s == 0u ? 1u : s;
}

// ------------------------------------------------------------------ ray
struct Ray {
    D3 o, d;
    Ray() {}
    Ray(const D3& oo, const D3& dd) : o(oo), d(dd.normalized()) {}   // rayo.h:21-24
};

// ------------------------------------------------------------------ primitives (primitiva.h)
bool hit_sphere(const TfgPrimitiva& p, const Ray& r, float& t) {
    D3 oc = r.o - D3(p.u.esfera.centro);
    float a = (float)r.d.dot(r.d);
    float b = (float)(2.0f * oc.dot(r.d));
    float c = (float)(oc.dot(oc) - p.u.esfera.radio * p.u.esfera.radio);
    float disc = b * b - 4.0f * a * c;
    if (disc < 0) return false;
    float sd = std::sqrt(disc);
    float t1 = (-b - sd) / (2.0f * a);
    float t2 = (-b + sd) / (2.0f * a);
    if (t1 > 1e-6f && t1 < t2) { t = t1; return true; }
    if (t2 > 1e-6f) { t = t2; return true; }
    return false;
}
bool hit_plane(const TfgPrimitiva& p, const Ray& r, float& t) {
    D3 n(p.u.plano.normal);
    float denom = (float)n.dot(r.d);
    if (std::fabs(denom) > 1e-6f) {
        D3 p0 = n * p.u.plano.distancia;
        t = (float)((p0 - r.o).dot(n) / denom);
        return t > 1e-6f;
    }
    return false;
}
bool hit_tri(const TfgPrimitiva& p, const Ray& r, float& t, float& u, float& v) {
    D3 v0(p.u.triangulo.v0), v1(p.u.triangulo.v1), v2(p.u.triangulo.v2);
    D3 e1 = v1 - v0, e2 = v2 - v0;
    D3 pv = r.d.cross(e2);
    float det = (float)e1.dot(pv);
    if (std::fabs(det) < 1e-6f) return false;
    float inv = 1.0f / det;
    D3 tvec = r.o - v0;
    u = (float)(tvec.dot(pv) * inv);
    if (u < 0.0f || u > 1.0f) return false;
    D3 q = tvec.cross(e1);
    v = (float)(r.d.dot(q) * inv);
    if (v < 0.0f || u + v > 1.0f) return false;
    t = (float)(e2.dot(q) * inv);
    return t > 1e-6f;
}
bool hit_prim(const TfgPrimitiva& p, const Ray& r, float& t, float& u, float& v) {
    if (p.tipo == TFG_TRIANGULO) return hit_tri(p, r, t, u, v);
    u = 0.0f; v = 0.0f;
    if (p.tipo == TFG_ESFERA) return hit_sphere(p, r, t);
    if (p.tipo == TFG_PLANO) return hit_plane(p, r, t);
    return false;
}

D3 prim_normal(const TfgPrimitiva& p, const D3& P, float u, float v) {   // escenario.h:123-142
    if (p.tipo == TFG_TRIANGULO) {
        D3 n0(p.u.triangulo.v0_normal), n1(p.u.triangulo.v1_normal), n2(p.u.triangulo.v2_normal);
        if (n0 != n1 || n0 != n2) {
            float b0 = 1.0f - u - v;
            D3 n = b0 * n0 + u * n1 + v * n2;
            float len = (float)std::sqrt(n.dot(n));
            if (len > 1e-6f) return n * (1.0f / len);
            return D3(0, 0, 0);
        }
        D3 v0(p.u.triangulo.v0);
        D3 n = (D3(p.u.triangulo.v1) - v0).cross(D3(p.u.triangulo.v2) - v0);
        if (n.dot(-P) < 0) n = n * -1.0f;
        return n.normalized();
    }
    if (p.tipo == TFG_ESFERA) return (P - D3(p.u.esfera.centro)).normalized();
    if (p.tipo == TFG_PLANO) return D3(p.u.plano.normal);
    return D3(0, 0, 0);
}

// ------------------------------------------------------------------ CWBVH traversal (traverse_cwbvh.cuh)
inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t bfind(uint32_t v) { return v ? 31u - (uint32_t)__builtin_clz(v) : 0xFFFFFFFFu; }
// prmt.b32 d, a, 0, 0xBA98: each result byte = sign of the matching byte of a, replicated.
inline uint32_t sign_extend_bytes(uint32_t a) {
    uint32_t r = 0;
    for (int k = 0; k < 4; ++k) if ((a >> (8 * k + 7)) & 1u) r |= 0xFFu << (8 * k);
    return r;
}
// vshl.u32.u32.u32.wrap.add d, a.bK, b.bK, c: (byte K of a) << (byte K of b mod 32), plus c.
inline uint32_t vshl_add(uint32_t a, uint32_t b, int k, uint32_t c) {
    uint32_t ab = (a >> (8 * k)) & 0xFFu, bb = (b >> (8 * k)) & 0xFFu;
    return (ab << (bb & 31u)) + c;
}
inline float qbyte(float f, int k) { return (float)((fbits(f) >> (8 * k)) & 0xFFu); }

struct Counts { uint32_t nodes = 0, plane_tests = 0, uv_tests = 0; };

// Returns (t, u, v, id) with id = 0xFFFFFFFF when nothing closer than t_max is hit.
void cwbvh_closest(const float* nodes_f, const float* tris_f, const float O[3], const float D[3], const float rD[3],
                   float t_max, float out[4], Counts* cnt) {
    uint32_t stack[2 * 64];
    uint32_t sp = 0, hit_addr = 0xFFFFFFFFu;
    float hu = 0.0f, hv = 0.0f, tcur = t_max;
    const uint32_t octinv4 = (7u - ((D[0] < 0 ? 4u : 0u) | (D[1] < 0 ? 2u : 0u) | (D[2] < 0 ? 1u : 0u))) * 0x1010101u;
    uint32_t ng_x = 0, ng_y = 0x80000000u, tg_x = 0, tg_y = 0;
    while (true) {
        if (ng_y > 0x00FFFFFFu) {
            const uint32_t hits = ng_y, imask = ng_y;
            const uint32_t bit = bfind(hits);
            const uint32_t base = ng_x;
            ng_y &= ~(1u << bit);
            if (ng_y > 0x00FFFFFFu) { stack[2 * sp] = ng_x; stack[2 * sp + 1] = ng_y; ++sp; }
            const uint32_t slot = (bit - 24u) ^ (octinv4 & 255u);
            const uint32_t rel = (uint32_t)__builtin_popcount(imask & ~(0xFFFFFFFFu << slot));
            const float* n = &nodes_f[(size_t)(base + rel) * 20];
            if (cnt) cnt->nodes++;
            const uint32_t ew = fbits(n[3]);
            ng_x = fbits(n[4]);
            tg_x = fbits(n[5]);
            tg_y = 0;
            uint32_t hitmask = 0;
            const float idir[3] = {bitsf((uint32_t)((int)(int8_t)(ew & 0xFF) + 127) << 23) * rD[0],
                                   bitsf((uint32_t)((int)(int8_t)((ew >> 8) & 0xFF) + 127) << 23) * rD[1],
                                   bitsf((uint32_t)((int)(int8_t)((ew >> 16) & 0xFF) + 127) << 23) * rD[2]};
            const float orig[3] = {(n[0] - O[0]) * rD[0], (n[1] - O[1]) * rD[1], (n[2] - O[2]) * rD[2]};
            // words: n2 = n[8..11], n3 = n[12..15], n4 = n[16..19]
            for (int half = 0; half < 2; ++half) {
                const uint32_t meta4 = fbits(n[6 + half]);
                const uint32_t inner4 = (meta4 & (meta4 << 1)) & 0x10101010u;
                const uint32_t inner_mask4 = sign_extend_bytes(inner4 << 3);
                const uint32_t bidx4 = (meta4 ^ (octinv4 & inner_mask4)) & 0x1F1F1F1Fu;
                const uint32_t cbits4 = (meta4 >> 5) & 0x07070707u;
                const float qlox = n[8 + half], qloy = n[10 + half], qloz = n[12 + half];
                const float qhix = n[14 + half], qhiy = n[16 + half], qhiz = n[18 + half];
                const float lox = rD[0] < 0 ? qhix : qlox, hix = rD[0] < 0 ? qlox : qhix;
                const float loy = rD[1] < 0 ? qhiy : qloy, hiy = rD[1] < 0 ? qloy : qhiy;
                const float loz = rD[2] < 0 ? qhiz : qloz, hiz = rD[2] < 0 ? qloz : qhiz;
                for (int k = 0; k < 4; ++k) {
                    const float tmin = std::fmax(std::fmax(std::fmax(std::fmaf(qbyte(lox, k), idir[0], orig[0]),
                                                                     std::fmaf(qbyte(loy, k), idir[1], orig[1])),
                                                           std::fmaf(qbyte(loz, k), idir[2], orig[2])), 0.0f);
                    const float tmax = std::fmin(std::fmin(std::fmin(std::fmaf(qbyte(hix, k), idir[0], orig[0]),
                                                                     std::fmaf(qbyte(hiy, k), idir[1], orig[1])),
                                                           std::fmaf(qbyte(hiz, k), idir[2], orig[2])), tcur);
                    if (tmin <= tmax) hitmask = vshl_add(cbits4, bidx4, k, hitmask);
                }
            }
            ng_y = (hitmask & 0xFF000000u) | (ew >> 24);
            tg_y = hitmask & 0x00FFFFFFu;
        } else {
            tg_x = ng_x; tg_y = ng_y;
            ng_x = 0; ng_y = 0;
        }
        while (tg_y != 0) {
            const uint32_t ti = bfind(tg_y);
            const uint32_t addr = tg_x + ti * 4u;
            const float* T0 = &tris_f[(size_t)addr * 4];
            const float* T1 = T0 + 4;
            const float* T2 = T0 + 8;
            const float* T3 = T0 + 12;
            if (cnt) cnt->plane_tests++;
            const float transS = T2[0] * O[0] + T2[1] * O[1] + T2[2] * O[2] + T2[3];
            const float transD = T2[0] * D[0] + T2[1] * D[1] + T2[2] * D[2];
            const float d = -transS / transD;
            tg_y -= 1u << ti;
            if (d <= 0.0f || d >= tcur) continue;
            if (cnt) cnt->uv_tests++;
            const float I[3] = {O[0] + d * D[0], O[1] + d * D[1], O[2] + d * D[2]};
            const float u = T0[0] * I[0] + T0[1] * I[1] + T0[2] * I[2] + T0[3];
            const float v = T1[0] * I[0] + T1[1] * I[1] + T1[2] * I[2] + T1[3];
            if (u >= 0.0f && v >= 0.0f && u + v < 1.0f) {
                hu = u; hv = v; tcur = d;
                hit_addr = fbits(T3[3]);
            }
        }
        if (ng_y <= 0x00FFFFFFu) {
            if (sp > 0) { --sp; ng_x = stack[2 * sp]; ng_y = stack[2 * sp + 1]; }
            else break;
        }
    }
    out[0] = tcur; out[1] = hu; out[2] = hv; out[3] = bitsf(hit_addr);
}

// ------------------------------------------------------------------ scene (escenario.h)
struct Scene {
    const TfgPrimitiva* prims; int nprims;
    const TfgLuzPuntual* lights; int nlights;
    const float* nodes; const float* tris; const TfgPrimitiva* mesh; int nmesh;
    int shadow_mesh;
};

// escenario.h:316-366 -- analytic primitives, then the CWBVH.
bool closest(const Scene& s, const Ray& r, float& t, const TfgPrimitiva** obj, float& u, float& v) {
    bool hit = false;
    float tmin = 1e9f;
    const TfgPrimitiva* best = nullptr;
    float ut = 0.0f, vt = 0.0f;
    for (int i = 0; i < s.nprims; ++i) {
        float tt, ul = 0.0f, vl = 0.0f;
        if (hit_prim(s.prims[i], r, tt, ul, vl) && tt < tmin && tt > 1e-6f) {
            tmin = tt; best = &s.prims[i]; ut = ul; vt = vl; hit = true;
        }
    }
    if (s.nodes && s.tris && s.nmesh > 0) {
        float O[3] = {(float)r.o.x, (float)r.o.y, (float)r.o.z};
        float D[3] = {(float)r.d.x, (float)r.d.y, (float)r.d.z};
        float rD[3] = {1.0f / D[0], 1.0f / D[1], 1.0f / D[2]};
        float h[4];
        cwbvh_closest(s.nodes, s.tris, O, D, rD, tmin, h, nullptr);
        uint32_t id = fbits(h[3]);
        if (id != 0xFFFFFFFFu && h[0] < tmin && h[0] > 1e-3f) {
            tmin = h[0]; ut = h[1]; vt = h[2]; best = &s.mesh[id]; hit = true;
        }
    }
    if (hit) { t = tmin; *obj = best; u = ut; v = vt; }
    return hit;
}

// Shadow query: escenario.h:248-290 with the reference kernel's null own-BVH
// (analytic primitives only); with shadow_mesh the CWBVH mesh is tested too.
bool shadow_closest(const Scene& s, const Ray& r, float& t) {
    bool hit = false;
    float tmin = 1e9f;
    for (int i = 0; i < s.nprims; ++i) {
        float tt, ul, vl;
        if (hit_prim(s.prims[i], r, tt, ul, vl) && tt < tmin && tt > 1e-6f) { tmin = tt; hit = true; }
    }
    if (s.shadow_mesh && s.nodes && s.tris && s.nmesh > 0) {
        float O[3] = {(float)r.o.x, (float)r.o.y, (float)r.o.z};
        float D[3] = {(float)r.d.x, (float)r.d.y, (float)r.d.z};
        float rD[3] = {1.0f / D[0], 1.0f / D[1], 1.0f / D[2]};
        float h[4];
        cwbvh_closest(s.nodes, s.tris, O, D, rD, tmin, h, nullptr);
        if (fbits(h[3]) != 0xFFFFFFFFu && h[0] < tmin && h[0] > 1e-3f) { tmin = h[0]; hit = true; }
    }
    if (hit) t = tmin;
    return hit;
}

C3 direct_light(const Scene& s, const D3& P, const D3& N, const TfgPrimitiva* obj) {   // escenario.h:144-184
    C3 L(0, 0, 0);
    for (int i = 0; i < s.nlights; ++i) {
        const TfgLuzPuntual& lz = s.lights[i];
        D3 dl = D3(lz.posicion) - P;
        float dist = (float)dl.length();
        dl = dl.normalized();
        float c = (float)N.dot(dl);
        if (c <= 0.0f) continue;
        Ray sr(P + dl * 1e-3f, dl);
        float ts;
        if (shadow_closest(s, sr, ts) && ts < dist) continue;
        C3 brdf = C3(obj->difuso) / (float)M_PI;
        dist = std::max(dist, 1.0f);
        C3 Li = C3(lz.intensidad) / (dist * dist);
        L = L + Li * brdf * c;
    }
    return L;
}

// ------------------------------------------------------------------ path (render.h)
struct PathOut {
    C3 color;
    bool need_inf = false; TfgDatosMLP inf{}; C3 thr_inf;
    bool save = false; TfgRegistroEntrenamiento reg{};
};

D3 reflect(const D3& d, const D3& n) { return (d - 2.0 * n * d.dot(n)).normalized(); }

D3 refract(const D3& d, const D3& n, double ior_obj, double& ior_cur) {
    D3 I = d.normalized(), N = n.normalized();
    double cosi = I.dot(N);
    cosi = std::fmax(-1.0, std::fmin(1.0, cosi));
    double etai = ior_cur, etat;
    if (cosi > 0.0) { N = -N; etat = 1.0; }
    else { cosi = -cosi; etat = ior_obj; }
    double eta = etai / etat;
    double k = 1.0 - eta * eta * (1.0 - cosi * cosi);
    if (k < 0.0) return reflect(I, N);
    ior_cur = etat;
    double cost = std::sqrt(k);
    D3 T = eta * I + (eta * cosi - cost) * N;
    return T.normalized();
}

D3 to_world(const D3& l, const D3& n) {
    D3 t;
    if (std::fabs(n.x) > std::fabs(n.y)) t = D3(n.z, 0, -n.x);
    else t = D3(0, -n.z, n.y);
    t.normalize();
    D3 b = n.cross(t);
    b.normalize();
    return l.x * t + l.y * b + l.z * n;
}

void set_geo(TfgDatosGeometricos& g, const D3& P, const D3& dir, const D3& n, const C3& kd, const C3& ks) {
    g.posicion = tv(P); g.direccion = tv(dir); g.normal = tv(n); g.difuso = tc(kd); g.especular = tc(ks);
}

void trace_path(const Scene& s, const TfgRenderParams& prm, Ray r0, uint32_t& rng, bool training, bool use_inf,
                PathOut& out) {
    C3 color(0, 0, 0), cam(1, 1, 1);
    Ray ray = r0;
    double ior = 1.0;
    C3 thr_train(0, 0, 0), pre(0, 0, 0);
    bool captured = false;
    float a0 = 0.0f, acur = 0.0f, asuf = 0.0f, apre = 0.0f;
    int depth = 0;
    float pdf_last = 1.0f;
    TfgRegistroEntrenamiento& reg = out.reg;
    std::memset(&reg, 0, sizeof(reg));
    bool save = false;
    const bool unbiased = training && (pcgf(rng) < 0.0625f);
    const float EPS = 1e-3f;
    const float PI = 3.14159265358979323846f;
    while (depth < prm.max_depth) {
        float t;
        const TfgPrimitiva* obj;
        float u = 0.0f, v = 0.0f;
        if (closest(s, ray, t, &obj, u, v)) {
            D3 P = ray.o + ray.d * t;
            D3 N = prim_normal(*obj, P, u, v);
            D3 view = -ray.d.normalized();
            float cos_t = (float)std::fabs(N.dot(-ray.d));
            bool dif = C3(obj->difuso).max() > EPS;
            bool spe = C3(obj->especular).max() > EPS;
            float dsq = t * t;
            if (depth == 0) {
                a0 = dsq / (4.0f * PI * std::fmax(cos_t, 1e-4f));
                acur = 0.0f;
            } else {
                float spread = dsq / (std::fmax(pdf_last, 1e-4f) * std::fmax(cos_t, 1e-4f));
                if (!captured) acur += spread;
                else asuf += spread;
            }
            bool foot_ok = acur >= a0 * 0.01f;
            C3 Le(obj->emision);
            if (Le.max() > 0.0f) {
                color = color + cam * Le;
                if (captured) {
                    set_geo(reg.tail, P, -ray.d.normalized(), N, C3(0, 0, 0), C3(0, 0, 0));
                    reg.luz_acumulada_sufijo = tc(color - pre);
                    reg.throughput_sufijo = tc(C3(0, 0, 0));
                    reg.factor_normalizacion = tc(thr_train);
                    reg.valido = 1;
                    save = true;
                }
                break;
            }
            if (dif) {
                D3 ps = P + N * EPS;
                C3 Ld = direct_light(s, ps, N, obj);
                color = color + cam * Ld;
            }
            if (captured) {
                bool stop = !unbiased && (asuf >= apre);
                C3 refl_t = C3(obj->difuso) + C3(obj->especular) + C3(obj->transmision);
                if (stop) {
                    D3 dm(view.x * 0.5f + 0.5f, view.y * 0.5f + 0.5f, view.z * 0.5f + 0.5f);
                    D3 nm(N.x * 0.5f + 0.5f, N.y * 0.5f + 0.5f, N.z * 0.5f + 0.5f);
                    set_geo(reg.tail, P, dm, nm, C3(obj->difuso), C3(obj->especular));
                    reg.luz_acumulada_sufijo = tc(color - pre);
                    reg.throughput_sufijo = tc(cam * refl_t);
                    reg.factor_normalizacion = tc(thr_train);
                    reg.valido = 1;
                    save = true;
                    break;
                }
            }
            if (dif && !spe && foot_ok) {
                C3 refl = C3(obj->difuso) + C3(obj->especular) + C3(obj->transmision);
                refl.r = std::fmax(refl.r, 1e-3f); refl.g = std::fmax(refl.g, 1e-3f); refl.b = std::fmax(refl.b, 1e-3f);
                D3 dm(view.x * 0.5f + 0.5f, view.y * 0.5f + 0.5f, view.z * 0.5f + 0.5f);
                D3 nm(N.x * 0.5f + 0.5f, N.y * 0.5f + 0.5f, N.z * 0.5f + 0.5f);
                if (!training && use_inf) {
                    TfgDatosMLP& d = out.inf;
                    std::memset(&d, 0, sizeof(d));
                    d.posicion = tv(P); d.direccion = tv(dm); d.normal = tv(nm);
                    d.difuso = obj->difuso; d.especular = obj->especular;
                    out.thr_inf = cam * refl;
                    out.need_inf = true;
                    break;
                } else if (training && !captured) {
                    set_geo(reg.head, P, dm, nm, C3(obj->difuso), C3(obj->especular));
                    thr_train = cam * refl;
                    pre = color;
                    apre = acur;
                    captured = true;
                }
            }
            // render.h:264-335
            {
                C3 kd(obj->difuso), ks(obj->especular), kt(obj->transmision);
                double mkd = kd.max(), mks = ks.max(), mkt = kt.max();
                double sum = mkd + mks + mkt;
                if (sum <= 0.0) {
                    cam = C3(0, 0, 0);
                } else {
                    double pd = mkd / sum, ps = mks / sum, pt = 1 - pd - ps;
                    double rb = pcgf(rng);
                    if (rb < pd) {
                        cam = cam * kd / (float)pd;
                        double r1 = pcgf(rng), r2 = pcgf(rng);
                        double phi = 2 * M_PI * r1;
                        double theta = std::acos(std::sqrt(1 - r2));
                        D3 wl(std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi), std::cos(theta));
                        if (!(wl.z <= EPS)) {
                            D3 wi = to_world(wl, N);
                            ray = Ray(P + wi * EPS, wi);
                            double c = std::fabs(wi.dot(N));
                            if (c < 1e-4) c = 1e-4;
                            pdf_last = (float)(c / PI);
                        }
                    } else if (rb < pd + ps) {
                        D3 w = reflect(ray.d, N);
                        cam = cam * ks / (float)ps;
                        ray = Ray(P + w * EPS, w);
                        pdf_last = 1e6f;
                    } else {
                        D3 w = refract(ray.d, N, obj->indice_refraccion, ior);
                        cam = cam * kt / (float)pt;
                        ray = Ray(P + w * EPS, w);
                        pdf_last = 1e6f;
                    }
                }
            }
            if (depth >= prm.rr_min_depth) {   // render.h:209-224
                double prob = std::fmax(cam.r, std::fmax(cam.g, cam.b));
                if (prob > 0.95) prob = 0.95;
                if (pcgf(rng) > prob) {
                    if (training && captured) {
                        reg.luz_acumulada_sufijo = tc(color - pre);
                        reg.throughput_sufijo = tc(C3(0, 0, 0));
                        reg.factor_normalizacion = tc(thr_train);
                        reg.valido = 1;
                        save = true;
                    }
                    break;
                }
                cam = cam / (float)prob;
            }
        } else {
            if (training && captured) {
                reg.luz_acumulada_sufijo = tc(color - pre);
                reg.throughput_sufijo = tc(C3(0, 0, 0));
                reg.factor_normalizacion = tc(thr_train);
                reg.valido = 1;
                save = true;
            }
            break;
        }
        depth++;
    }
    if (training && captured && !save) {
        reg.luz_acumulada_sufijo = tc(color - pre);
        reg.throughput_sufijo = tc(C3(0, 0, 0));
        reg.factor_normalizacion = tc(thr_train);
        reg.valido = 1;
        save = true;
    }
    if (training && captured) {
        color = pre;
        out.need_inf = true;
        TfgDatosMLP& d = out.inf;
        std::memset(&d, 0, sizeof(d));
        d.posicion = reg.head.posicion; d.direccion = reg.head.direccion; d.normal = reg.head.normal;
        d.difuso = reg.head.difuso; d.especular = reg.head.especular;
        out.thr_inf = thr_train;
    }
    out.save = save;
    out.color = color;
}

// camara.h:42-59
Ray camera_ray(const TfgCamara& c, int x, int y, int W, int H, float ox, float oy) {
    float u = (x + ox) / W;
    float v = (y + oy) / H;
    float px = (2.0f * u - 1.0f) * (c.ancho_plano * 0.5f);
    float py = (1.0f - 2.0f * v) * (c.alto_plano * 0.5f);
    D3 pos(c.posicion);
    D3 pp = pos + D3(c.frente) * c.distancia_focal + D3(c.izquierda) * px + D3(c.arriba) * py;
    D3 dir = (pp - pos).normalized();
    return Ray(pos, dir);
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

uint32_t orc_seed(int px, int py, int frame) { return seed(px, py, frame); }

void orc_pcg_stream(uint32_t state, int n, uint32_t* out_u32, float* out_f) {
    for (int i = 0; i < n; ++i) {
        uint32_t s = state;
        out_f[i] = pcgf(s);
        out_u32[i] = pcg(state);
    }
}

// Closest hits of n rays (8 floats each: O, t_max, D, -) with 1/D per ray
// (escenario.h:339-341).  counts: 3 uint32 per ray (nodes, plane tests, uv tests).
void orc_trace_batch(const float* nodes, const float* tris_ref, const float* rays, int n, float* hits,
                     uint32_t* counts, int nthreads) {
    auto work = [&](int lo, int hi) {
        for (int i = lo; i < hi; ++i) {
            const float* r = &rays[8 * (size_t)i];
            float O[3] = {r[0], r[1], r[2]}, D[3] = {r[4], r[5], r[6]};
            float rD[3] = {1.0f / D[0], 1.0f / D[1], 1.0f / D[2]};
            Counts c;
            cwbvh_closest(nodes, tris_ref, O, D, rD, r[3], &hits[4 * (size_t)i], &c);
            if (counts) { counts[3 * (size_t)i] = c.nodes; counts[3 * (size_t)i + 1] = c.plane_tests; counts[3 * (size_t)i + 2] = c.uv_tests; }
        }
    };
    nthreads = std::max(1, nthreads);
    std::vector<std::thread> th;
    int chunk = (n + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
        int lo = k * chunk, hi = std::min(n, lo + chunk);
        if (lo < hi) th.emplace_back(work, lo, hi);
    }
    for (auto& t : th) t.join();
}

// Brute force over the reference triangle layout (same test, every triangle,
// in BVH order).  Used to check the builder: the BVH must find this hit.
void orc_brute_batch(const float* tris_ref, uint32_t ntris, const float* rays, int n, float* hits, int nthreads) {
    auto work = [&](int lo, int hi) {
        for (int i = lo; i < hi; ++i) {
            const float* r = &rays[8 * (size_t)i];
            const float O[3] = {r[0], r[1], r[2]}, D[3] = {r[4], r[5], r[6]};
            float tcur = r[3], hu = 0, hv = 0;
            uint32_t id = 0xFFFFFFFFu;
            for (uint32_t k = 0; k < ntris; ++k) {
                const float* T0 = &tris_ref[16 * (size_t)k];
                const float* T1 = T0 + 4;
                const float* T2 = T0 + 8;
                const float transS = T2[0] * O[0] + T2[1] * O[1] + T2[2] * O[2] + T2[3];
                const float transD = T2[0] * D[0] + T2[1] * D[1] + T2[2] * D[2];
                const float d = -transS / transD;
                if (d <= 0.0f || d >= tcur) continue;
                const float I[3] = {O[0] + d * D[0], O[1] + d * D[1], O[2] + d * D[2]};
                const float u = T0[0] * I[0] + T0[1] * I[1] + T0[2] * I[2] + T0[3];
                const float v = T1[0] * I[0] + T1[1] * I[1] + T1[2] * I[2] + T1[3];
                if (u >= 0.0f && v >= 0.0f && u + v < 1.0f) { tcur = d; hu = u; hv = v; id = fbits(T0[15]); }
            }
            float* h = &hits[4 * (size_t)i];
            h[0] = tcur; h[1] = hu; h[2] = hv; h[3] = bitsf(id);
        }
    };
    nthreads = std::max(1, nthreads);
    std::vector<std::thread> th;
    int chunk = (n + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
        int lo = k * chunk, hi = std::min(n, lo + chunk);
        if (lo < hi) th.emplace_back(work, lo, hi);
    }
    for (auto& t : th) t.join();
}

// Camera rays in the reference's arithmetic (double), rounded to float, in the
// 8-float layout; rows [y0, y1).
void orc_camera_rays(const TfgCamara* cam, int W, int H, int frame, int y0, int y1, float* rays) {
    for (int y = y0; y < y1; ++y)
        for (int x = 0; x < W; ++x) {
            uint32_t rng = seed(x, y, frame);
            float ox = pcgf(rng), oy = pcgf(rng);
            Ray r = camera_ray(*cam, x, y, W, H, ox, oy);
            float* o = &rays[8 * ((size_t)(y - y0) * W + x)];
            o[0] = (float)r.o.x; o[1] = (float)r.o.y; o[2] = (float)r.o.z; o[3] = 1e9f;
            o[4] = (float)r.d.x; o[5] = (float)r.d.y; o[6] = (float)r.d.z; o[7] = 0.0f;
        }
}

// One sample per pixel of rows [y0, y1) (render.h:416-466).  img: 3 floats per
// pixel of the row range.  Optional per-pixel NRC outputs (row-range indexed):
// infer / thr (written as the reference writes them) and regs with
// reg_flags[p] = 1 where the reference would append a training record.
void orc_render(const TfgPrimitiva* prims, int nprims, const TfgLuzPuntual* lights, int nlights, const float* nodes,
                const float* tris_ref, const TfgPrimitiva* mesh, int nmesh, const TfgCamara* cam, int W, int H,
                int frame, const TfgRenderParams* prm, int y0, int y1, float* img, TfgDatosMLP* infer,
                TfgColor* thr, TfgRegistroEntrenamiento* regs, uint8_t* reg_flags, int use_inf, int train,
                int nthreads) {
    Scene s{prims, nprims, lights, nlights, nodes, tris_ref, mesh, nmesh, prm->shadow_mesh};
    std::atomic<int> next_row(y0);
    auto work = [&]() {
        while (true) {
            int y = next_row.fetch_add(1);
            if (y >= y1) break;
            for (int x = 0; x < W; ++x) {
                uint32_t rng = seed(x, y, frame);
                float ox = pcgf(rng), oy = pcgf(rng);
                Ray r = camera_ray(*cam, x, y, W, H, ox, oy);
                bool training = train ? (use_inf ? (pcgf(rng) < 0.05f) : true) : false;
                PathOut po;
                trace_path(s, *prm, r, rng, training, use_inf != 0, po);
                size_t p = (size_t)(y - y0) * W + x;
                img[3 * p] = po.color.r; img[3 * p + 1] = po.color.g; img[3 * p + 2] = po.color.b;
                if (thr) {
                    if (po.need_inf) { if (infer) infer[p] = po.inf; thr[p] = tc(po.thr_inf); }
                    else thr[p] = TfgColor{0, 0, 0};
                }
                if (reg_flags) {
                    reg_flags[p] = (training && po.save) ? 1 : 0;
                    if (regs && reg_flags[p]) regs[p] = po.reg;
                }
            }
        }
    };
    nthreads = std::max(1, nthreads);
    std::vector<std::thread> th;
    for (int k = 0; k < nthreads; ++k) th.emplace_back(work);
    for (auto& t : th) t.join();
}

// ------------------------------------------------------------------ small kernels
void orc_indices(int* idx, int max_range, int count, uint32_t sd) {   // NrcKernel.cu:10-16
    for (int i = 0; i < count; ++i) { uint32_t s = sd ^ (uint32_t)i; idx[i] = (int)(pcg(s) % (uint32_t)max_range); }
}

static float unit_clamp(float v, float lo, float hi) {   // NrcKernel.cu:5-8
    float n = (v - lo) / (hi - lo);
    return std::fmin(std::fmax(n, 0.0f), 1.0f);
}

static void row15(const TfgDatosMLP& d, const TfgSceneBounds& b, float* r) {
    r[0] = unit_clamp((float)d.posicion.x, (float)b.min.x, (float)b.max.x);
    r[1] = unit_clamp((float)d.posicion.y, (float)b.min.y, (float)b.max.y);
    r[2] = unit_clamp((float)d.posicion.z, (float)b.min.z, (float)b.max.z);
    r[3] = (float)d.direccion.x; r[4] = (float)d.direccion.y; r[5] = (float)d.direccion.z;
    r[6] = (float)d.normal.x; r[7] = (float)d.normal.y; r[8] = (float)d.normal.z;
    r[9] = d.difuso.r; r[10] = d.difuso.g; r[11] = d.difuso.b;
    r[12] = d.especular.r; r[13] = d.especular.g; r[14] = d.especular.b;
}

void orc_train_rows(const TfgDatosMLP* buf, const int* idx, int batch, int n_in, int n_out, const TfgSceneBounds* b,
                    float* in, float* tgt) {   // NrcKernel.cu:18-68
    for (int i = 0; i < batch; ++i) {
        const TfgDatosMLP& d = buf[idx[i]];
        row15(d, *b, in + (size_t)i * n_in);
        float c[3] = {d.color.r, d.color.g, d.color.b};
        for (int k = 0; k < 3; ++k) if (c[k] > 100000.0f) c[k] = 100000.0f;
        for (int k = 0; k < 3; ++k) tgt[(size_t)i * n_out + k] = c[k];
    }
}

void orc_infer_rows(const TfgDatosMLP* d, int n, int n_in, float* out, const TfgSceneBounds* b) {   // NrcKernel.cu:70-97
    for (int i = 0; i < n; ++i) row15(d[i], *b, out + (size_t)i * n_in);
}

void orc_scrub(const float* net, TfgColor* out, int n) {   // NrcKernel.cu:99-126
    for (int i = 0; i < n; ++i) {
        float c[3] = {net[3 * i], net[3 * i + 1], net[3 * i + 2]};
        for (int k = 0; k < 3; ++k) {
            if (c[k] < 0.0f) c[k] = 0.0f;
            if (std::isnan(c[k])) c[k] = 0.0f;
            if (c[k] > 100000.0f) c[k] = 100000.0f;
            if (std::isinf(c[k])) c[k] = 100000.0f;
        }
        out[i] = TfgColor{c[0], c[1], c[2]};
    }
}

void orc_composite(TfgColor* img, const TfgColor* pred, const TfgColor* thr, int n) {   // RenderKernel.cu:49-66
    for (int i = 0; i < n; ++i) {
        C3 f(img[i]), t(thr[i]), p(pred[i]);
        if (t.r > 0 || t.g > 0 || t.b > 0) f = f + (t * p);
        img[i] = tc(f);
    }
}

// Final image: sum * (1 / frames) (main.cpp:1106-1110), the filmic curve
// (imagen.h:193-204) and the 8-bit conversion of guardarPNG
// (imagen_utils.h:59-62); float arithmetic in the written order.
static float orc_filmic(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    x = x * 0.6f;
    const float v = (x * (a * x + b)) / (x * (c * x + d) + e);
    return std::min(std::max(v, 0.0f), 1.0f);
}

void orc_tonemap_filmic(const float* sum, int frames, int n, float* hdr, uint8_t* rgb8) {
    const float inv = 1.0f / (float)frames;
    for (int i = 0; i < 3 * n; ++i) {
        const float v = sum[i] * inv;
        hdr[i] = v;
        rgb8[i] = (uint8_t)std::round(std::min(std::max(orc_filmic(v), 0.0f), 1.0f) * 255.0f);
    }
}

void orc_targets(const TfgRegistroEntrenamiento* regs, const TfgColor* tail, TfgDatosMLP* out, int n) {   // RenderKernel.cu:92-137
    for (int i = 0; i < n; ++i) {
        const TfgRegistroEntrenamiento& r = regs[i];
        if (!r.valido) { out[i].color = TfgColor{0, 0, 0}; continue; }
        C3 tot = C3(r.luz_acumulada_sufijo) + (C3(r.throughput_sufijo) * C3(tail[i]));
        C3 den(r.factor_normalizacion);
        float c[3] = {tot.r / std::fmax(den.r, 1e-8f), tot.g / std::fmax(den.g, 1e-8f), tot.b / std::fmax(den.b, 1e-8f)};
        for (int k = 0; k < 3; ++k) {
            c[k] = std::fmin(c[k], 100000.0f);
            if (std::isnan(c[k]) || std::isinf(c[k])) c[k] = 0.0f;
        }
        TfgDatosMLP d;
        d.posicion = r.head.posicion; d.direccion = r.head.direccion; d.normal = r.head.normal;
        d.difuso = r.head.difuso; d.especular = r.head.especular; d.color = TfgColor{c[0], c[1], c[2]};
        out[i] = d;
    }
}

void orc_tail(const TfgRegistroEntrenamiento* regs, TfgDatosMLP* out, int n) {   // RenderKernel.cu:139-166
    for (int i = 0; i < n; ++i) {
        TfgDatosMLP d;
        std::memset(&d, 0, sizeof(d));
        if (regs[i].valido) {
            d.posicion = regs[i].tail.posicion; d.direccion = regs[i].tail.direccion; d.normal = regs[i].tail.normal;
            d.difuso = regs[i].tail.difuso; d.especular = regs[i].tail.especular;
        }
        out[i] = d;
    }
}

void orc_default_camera(TfgCamara* c, int W, int H) {   // RenderKernel.cu:68-90, camara.h:29-40
    float focal = 1.0f, fovd = 45.0f;
    float fov = fovd * M_PI / 180.0f;
    float alto = 2.0f * focal * std::tan(fov / 2.0f);
    float ancho = alto * (static_cast<float>(W) / H);
    D3 f = D3(0, 0, -1).normalized(), a = D3(0, 1, 0).normalized();
    D3 l = f.cross(a).normalized();
    a = l.cross(f).normalized();
    c->posicion = TfgVec3d{0, -0.75, 4.25};
    c->frente = tv(f); c->arriba = tv(a); c->izquierda = tv(l);
    c->ancho_plano = ancho; c->alto_plano = alto; c->distancia_focal = focal;
}

}  // extern "C"
