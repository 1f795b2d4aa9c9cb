// Device helpers shared by the wavefront stages: float3 arithmetic, the
// reference's PCG-style RNG, the pinhole camera, analytic primitive tests
// and the shading formulas.  Each function names the reference code whose
// results it reproduces; arithmetic is FP32 except the camera ray, which is
// built in FP64 like the reference (camara.h:42-59) and then rounded.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tfg_pt.h"
#include "tfg_runtime.h"

namespace tfg {

// ---------------------------------------------------------------- layout
static_assert(sizeof(TfgVec3d) == 24, "Vector3d is 24 B");
static_assert(sizeof(TfgColor) == 12, "Color is 12 B");
static_assert(sizeof(TfgPrimitiva) == 200, "Primitiva is 200 B");
static_assert(offsetof(TfgPrimitiva, u) == 56, "Primitiva union at offset 56");
static_assert(sizeof(TfgLuzPuntual) == 40, "LuzPuntual is 40 B");
static_assert(sizeof(TfgCamara) == 112, "Camara is 112 B");
static_assert(sizeof(TfgDatosMLP) == 112, "DatosMLP is 112 B");
static_assert(sizeof(TfgDatosGeometricos) == 96, "DatosGeometricos is 96 B");
static_assert(sizeof(TfgRegistroEntrenamiento) == 232, "RegistroEntrenamiento is 232 B");
static_assert(offsetof(TfgRegistroEntrenamiento, valido) == 228, "valido at 228");
static_assert(sizeof(TfgSceneBounds) == 48, "SceneBounds is 48 B");
static_assert(sizeof(TfgImagenGPU) == 16, "ImagenGPU is 16 B");
static_assert(sizeof(TfgTinyBVHD_GPU) == 24, "TinyBVHD_GPU is 24 B");

constexpr float kEps = 1e-3f;                       // render.h:27, escenario.h:40
constexpr float kPiF = 3.14159265358979323846f;     // render.h:20

// Cell of the radiance cache's gate grid (kGateRes per axis over the scene
// bounds: cell = floor((x - lo) * inv)) holding a point; points outside the
// bounds fall into the border cells.  The render pass reads the cell's gate
// bit with it and the gate update adds a record's error to it.
__device__ __forceinline__ uint32_t gate_cell(const float (&lo)[3], const float (&inv)[3], float x, float y,
                                              float z) {
    const int r = kGateRes - 1;
    const int ix = min(max(__float2int_rd((x - lo[0]) * inv[0]), 0), r);
    const int iy = min(max(__float2int_rd((y - lo[1]) * inv[1]), 0), r);
    const int iz = min(max(__float2int_rd((z - lo[2]) * inv[2]), 0), r);
    return ((uint32_t)iz * kGateRes + (uint32_t)iy) * kGateRes + (uint32_t)ix;
}

// ---------------------------------------------------------------- float3
struct V3 {
    float x, y, z;
};
__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 normalized(V3 a) {
    float l = sqrtf(dot(a, a));
    return l > 0.0f ? a * (1.0f / l) : a;   // vector3d.h:65-71 leaves a zero vector unchanged
}
// Color / float (color.h:40-46): division by zero gives black.
__device__ __forceinline__ V3 div_or_black(V3 c, float s) {
    return s == 0.0f ? v3(0.0f, 0.0f, 0.0f) : v3(c.x / s, c.y / s, c.z / s);
}
__device__ __forceinline__ float cmax(V3 c) {   // color.h:66-78 (r >= g ? r : g, then b)
    float m = c.x >= c.y ? c.x : c.y;
    return c.z > m ? c.z : m;
}
__device__ __forceinline__ V3 ld3(const TfgColor& c) { return v3(c.r, c.g, c.b); }
__device__ __forceinline__ V3 ld3(const TfgVec3d& v) { return v3((float)v.x, (float)v.y, (float)v.z); }

// ---------------------------------------------------------------- RNG
// rng.h:12-17: LCG step followed by an xorshift-multiply output permutation.
__host__ __device__ __forceinline__ uint32_t pcg_next(uint32_t& s) {
    s = s * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
// rng.h:20-22: u32 -> float (round to nearest) times 2^-32; can return 1.0f.
__device__ __forceinline__ float pcg_uniform(uint32_t& s) {
    return __uint2float_rn(pcg_next(s)) * (1.0f / 4294967296.0f);
}
// rng.h:25-35: pixel/frame seed mixed with Wang's integer hash; 0 maps to 1.
__host__ __device__ __forceinline__ uint32_t seed_pixel(int px, int py, int frame) {
    uint32_t s = ((uint32_t)py << 16) | ((uint32_t)px & 0xFFFFu);
    s ^= (uint32_t)frame * 719393u;
    s = (s ^ 61u) ^ (s >> 16u);
    s *= 0x27d4eb2du;
    s = s ^ (s >> 15u);
    return s == 0u ? 1u : s;
}

// ---------------------------------------------------------------- camera
// camara.h:42-59 in FP64, then rounded to FP32 (escenario.h:339-341 rounds the
// same way before traversal).  Rayo's constructor normalises again
// (rayo.h:21-24), which is reproduced.
__device__ __forceinline__ void camera_ray(const TfgCamara& c, int x, int y, int W, int H, float ox, float oy,
                                           V3& O, V3& D) {
    float u = (x + ox) / W;
    float v = (y + oy) / H;
    float px = (2.0f * u - 1.0f) * (c.ancho_plano * 0.5f);
    float py = (1.0f - 2.0f * v) * (c.alto_plano * 0.5f);
    double fx = c.posicion.x + c.frente.x * (double)c.distancia_focal + c.izquierda.x * (double)px + c.arriba.x * (double)py;
    double fy = c.posicion.y + c.frente.y * (double)c.distancia_focal + c.izquierda.y * (double)px + c.arriba.y * (double)py;
    double fz = c.posicion.z + c.frente.z * (double)c.distancia_focal + c.izquierda.z * (double)px + c.arriba.z * (double)py;
    double dx = fx - c.posicion.x, dy = fy - c.posicion.y, dz = fz - c.posicion.z;
    for (int k = 0; k < 2; ++k) {
        double l = sqrt(dx * dx + dy * dy + dz * dz);
        if (l > 0.0) { double il = 1.0 / l; dx *= il; dy *= il; dz *= il; }
    }
    O = v3((float)c.posicion.x, (float)c.posicion.y, (float)c.posicion.z);
    D = v3((float)dx, (float)dy, (float)dz);
}

// ---------------------------------------------------------------- analytic primitives
// FP32 copy of an analytic primitive, prepared once per block.
struct APrim {
    int tipo;          // TFG_ESFERA / TFG_PLANO / TFG_TRIANGULO
    float a[9];        // sphere: c.xyz, r;  plane: n.xyz, dist;  triangle: v0, v1, v2
};

__device__ __forceinline__ void aprim_load(const TfgPrimitiva& p, APrim& q) {
    q.tipo = p.tipo;
    if (p.tipo == TFG_ESFERA) {
        q.a[0] = (float)p.u.esfera.centro.x; q.a[1] = (float)p.u.esfera.centro.y; q.a[2] = (float)p.u.esfera.centro.z;
        q.a[3] = p.u.esfera.radio;
    } else if (p.tipo == TFG_PLANO) {
        q.a[0] = (float)p.u.plano.normal.x; q.a[1] = (float)p.u.plano.normal.y; q.a[2] = (float)p.u.plano.normal.z;
        q.a[3] = p.u.plano.distancia;
    } else {
        q.a[0] = (float)p.u.triangulo.v0.x; q.a[1] = (float)p.u.triangulo.v0.y; q.a[2] = (float)p.u.triangulo.v0.z;
        q.a[3] = (float)p.u.triangulo.v1.x; q.a[4] = (float)p.u.triangulo.v1.y; q.a[5] = (float)p.u.triangulo.v1.z;
        q.a[6] = (float)p.u.triangulo.v2.x; q.a[7] = (float)p.u.triangulo.v2.y; q.a[8] = (float)p.u.triangulo.v2.z;
    }
}

// primitiva.h:121-200: sphere (nearer root above 1e-6), plane (|denom| > 1e-6),
// Moller-Trumbore triangle (|det| >= 1e-6, t > 1e-6).  u,v = weights of v1,v2.
__device__ __forceinline__ bool aprim_hit(const APrim& q, V3 O, V3 D, float& t, float& u, float& v) {
    u = 0.0f; v = 0.0f;
    if (q.tipo == TFG_ESFERA) {
        V3 oc = O - v3(q.a[0], q.a[1], q.a[2]);
        float a = dot(D, D);
        float b = 2.0f * dot(oc, D);
        float c = dot(oc, oc) - q.a[3] * q.a[3];
        float disc = b * b - 4.0f * a * c;
        if (disc < 0.0f) return false;
        float sd = sqrtf(disc);
        float t1 = (-b - sd) / (2.0f * a);
        float t2 = (-b + sd) / (2.0f * a);
        if (t1 > 1e-6f && t1 < t2) { t = t1; return true; }
        if (t2 > 1e-6f) { t = t2; return true; }
        return false;
    } else if (q.tipo == TFG_PLANO) {
        V3 n = v3(q.a[0], q.a[1], q.a[2]);
        float denom = dot(n, D);
        if (fabsf(denom) > 1e-6f) {
            V3 p0 = n * q.a[3];
            t = dot(p0 - O, n) / denom;
            return t > 1e-6f;
        }
        return false;
    } else if (q.tipo == TFG_TRIANGULO) {
        V3 v0 = v3(q.a[0], q.a[1], q.a[2]);
        V3 e1 = v3(q.a[3], q.a[4], q.a[5]) - v0;
        V3 e2 = v3(q.a[6], q.a[7], q.a[8]) - v0;
        V3 pv = cross(D, e2);
        float det = dot(e1, pv);
        if (fabsf(det) < 1e-6f) return false;
        float inv = 1.0f / det;
        V3 tv = O - v0;
        u = dot(tv, pv) * inv;
        if (u < 0.0f || u > 1.0f) return false;
        V3 qv = cross(tv, e1);
        v = dot(D, qv) * inv;
        if (v < 0.0f || u + v > 1.0f) return false;
        t = dot(e2, qv) * inv;
        return t > 1e-6f;
    }
    return false;
}

// ---------------------------------------------------------------- material / normal
struct Material {
    V3 emision, difuso, especular, transmision;
    float ior;
};
__device__ __forceinline__ Material load_material(const TfgPrimitiva* p) {
    Material m;
    m.emision = ld3(p->emision);
    m.difuso = ld3(p->difuso);
    m.especular = ld3(p->especular);
    m.transmision = ld3(p->transmision);
    m.ior = p->indice_refraccion;
    return m;
}

// escenario.h:123-142 with primitiva.h:84-101 (smooth) and :202-220 (flat):
// triangles with differing vertex normals are shaded with the barycentric
// normal, others with the face normal turned toward the world origin; spheres
// use (p - c)/|p - c|; planes use the stored normal as is (not renormalised).
__device__ __forceinline__ V3 surface_normal(const TfgPrimitiva* p, V3 P, float u, float v) {
    if (p->tipo == TFG_TRIANGULO) {
        const TfgVec3d& n0 = p->u.triangulo.v0_normal;
        const TfgVec3d& n1 = p->u.triangulo.v1_normal;
        const TfgVec3d& n2 = p->u.triangulo.v2_normal;
        bool smooth = (n0.x != n1.x || n0.y != n1.y || n0.z != n1.z) || (n0.x != n2.x || n0.y != n2.y || n0.z != n2.z);
        if (smooth) {
            float b0 = 1.0f - u - v;
            V3 n = ld3(n0) * b0 + ld3(n1) * u + ld3(n2) * v;
            float len = sqrtf(dot(n, n));
            if (len > 1e-6f) return n * (1.0f / len);
            return v3(0.0f, 0.0f, 0.0f);
        }
        V3 a = ld3(p->u.triangulo.v0);
        V3 n = cross(ld3(p->u.triangulo.v1) - a, ld3(p->u.triangulo.v2) - a);
        if (dot(n, -P) < 0.0f) n = n * -1.0f;
        return normalized(n);
    }
    if (p->tipo == TFG_ESFERA) return normalized(P - ld3(p->u.esfera.centro));
    if (p->tipo == TFG_PLANO) return ld3(p->u.plano.normal);
    return v3(0.0f, 0.0f, 0.0f);
}

// render.h:396-413: orthonormal frame around n (n is not renormalised).
__device__ __forceinline__ V3 to_world(V3 l, V3 n) {
    V3 t = fabsf(n.x) > fabsf(n.y) ? v3(n.z, 0.0f, -n.x) : v3(0.0f, -n.z, n.y);
    t = normalized(t);
    V3 b = normalized(cross(n, t));
    return t * l.x + b * l.y + n * l.z;
}

// render.h:337-340.
__device__ __forceinline__ V3 reflect_dir(V3 d, V3 n) { return normalized(d - n * (2.0f * dot(d, n))); }

// render.h:342-376 (Snell with total internal reflection; updates the medium IOR).
__device__ __forceinline__ V3 refract_dir(V3 d, V3 n, float ior_obj, float& ior_cur) {
    V3 I = normalized(d);
    V3 N = normalized(n);
    float cosi = fmaxf(-1.0f, fminf(1.0f, dot(I, N)));
    float etai = ior_cur, etat;
    if (cosi > 0.0f) { N = -N; etat = 1.0f; }
    else { cosi = -cosi; etat = ior_obj; }
    float eta = etai / etat;
    float k = 1.0f - eta * eta * (1.0f - cosi * cosi);
    if (k < 0.0f) return reflect_dir(I, N);
    ior_cur = etat;
    float cost = sqrtf(k);
    return normalized(I * eta + N * (eta * cosi - cost));
}

}  // namespace tfg
