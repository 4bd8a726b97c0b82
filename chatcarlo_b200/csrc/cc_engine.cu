// chatcarlo_b200 engine: photon transport for 1-150 keV on sm_100a.
//
// One persistent kernel runs the event loop of ChatCarlo's
// transport_photons (chatcarlo/transport.py:98-233).  Every lane owns one
// photon; when its history ends the lane takes the next history from a
// warp-local pool that the warp refills from a global counter, so lanes
// never wait for the longest history of their warp.  Per step a lane
//   * finds its material at the segment start (geometry.py:205-212),
//   * looks up mu in the material's union energy grid (materials.py:228-289),
//   * finds the next analytic boundary (geometry.py:214-231),
//   * decides between crossing and interacting with its optical depth tau
//     (transport.py:137-158),
//   * walks the segment through the voxel grid, scoring E*mu_en and
//     h*(10)/Phi times the exact overlap length (tally.py:248-293 scores
//     the same expectation with stratified points),
//   * samples photoelectric absorption with K fluorescence, bound Compton
//     or Rayleigh scattering (physics.py:95-367).
// Tracking and sampling are FP32; tallies and the collision estimator are
// FP64.  Batches of histories score into separate scratch grids that a
// fold kernel turns into the batch statistics of VoxelGrid.end_batch
// (tally.py:59-94).
#include <math_constants.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <math.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "philox.cuh"
#include "../../include/chatcarlo_b200.h"

namespace cc {

constexpr int MAX_PRIMS = 64;
constexpr int MAX_MATS = 16;
constexpr int MAX_ELEMS_PER_MAT = 16;
constexpr int MAX_ELEMS = 48;
constexpr int TABLE_N = 2000;            // F, A, S tables (materials.py:376-496)
constexpr int N_BUCKETS = 4096;          // uniform log-E index per material
constexpr int RAY_BUCKETS = 1024;        // uniform-in-A index of each Rayleigh A(x) table
constexpr int MAX_SCRATCH = 64;          // batches per launch
// status bits
constexpr unsigned ST_ENERGY = 1u, ST_RAYLEIGH_Q = 2u, ST_STEPS = 4u, ST_BOUNDS = 8u;

// Precision.  The engine tracks and samples in FP32: positions, directions,
// distances, energies, optical depths, cross-section lookups and the
// samplers' arithmetic (tallies and the collision estimator are FP64
// either way).  A second build of this file with -DCC_TRACK_FP64 does all of
// that in FP64, with FP64 tables and the same random numbers (each 32-bit
// draw turned into an FP64 uniform), and without fast-math intrinsics: the
// FP64 reference against which every tally's cost of FP32 is measured.
// P(x) is a floating literal of the build's precision.
#ifdef CC_TRACK_FP64
typedef double real;
typedef double phys;
struct __align__(16) PNode { double x, y, z, w; };
#define P(x) x
#else
typedef float real;
typedef float phys;
typedef float4 PNode;
#define P(x) x##f
#endif
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float p_log(float x) { return __logf(x); }
__device__ __forceinline__ double p_log(double x) { return log(x); }
__device__ __forceinline__ float p_exp(float x) { return __expf(x); }
__device__ __forceinline__ double p_exp(double x) { return exp(x); }
__device__ __forceinline__ void p_sincos(float x, float* s, float* c) { __sincosf(x, s, c); }
__device__ __forceinline__ void p_sincos(double x, double* s, double* c) { sincos(x, s, c); }
__device__ __forceinline__ PNode ldg_node(const PNode* p) {
#ifdef CC_TRACK_FP64
    const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return PNode{a.x, a.y, b.x, b.y};
#else
    return __ldg(p);
#endif
}
// a uniform draw in (0, 1] of the build's precision from the next 32 bits
__device__ __forceinline__ phys uni(HistoryRng& r) {
#ifdef CC_TRACK_FP64
    return r.uniform_d();
#else
    return r.uniform();
#endif
}

constexpr phys E_MIN_KEV = P(1.0);
constexpr phys E_MAX_KEV = P(150.0);
constexpr phys HC = P(12.3984193);        // keV Angstrom (physics.py:35)
constexpr phys MEC2 = P(511.0);           // keV (physics.py:34)
constexpr phys FLUOR_CUTOFF = P(5.0);     // keV (physics.py:38)
constexpr phys TWO_PI = P(6.283185307179586);

struct DevPrim {
    int type, material, axis, pad;
    real c[3];
    real h[3];      // box half sizes, ellipsoid semi-axes
    real r2;        // radius^2
    real r;         // radius; ellipsoid: 1 / smallest semi-axis
    real hh;        // cylinder half height
};

struct DevMaterial {
    phys density;
    int n_nodes, n_el, node_off;
    int elem_off, bucket_off;
    phys bucket_scale;
    int el_slot[MAX_ELEMS_PER_MAT];
};

struct DevElement {
    phys k_edge, k_prob, omega;
    int n_lines, emits, z;
    phys ray_scale;        // RAY_BUCKETS / A(x_end)
    phys line_e[8];
    phys line_cum[8];
};

struct KTables {
    const PNode* nodes;        // 2 per node: {ln E, ln photo, ln Compton, ln Rayleigh}, {ln total, ln mu_en, ln h10, 0}
    const phys* elem_cum;      // per material [3][n_el - 1][n_nodes] normalised cumulative element weights
    const unsigned short* bucket;
    const DevMaterial* mats;
    const DevElement* elems;
    const phys* sq;       // [n_elem][TABLE_N] S/Z
    const phys* rx;       // [n_elem][TABLE_N]
    const phys* ra;       // [n_elem][TABLE_N]
    const int* ray_bucket; // [n_elem][RAY_BUCKETS + 1] last row with A <= bucket start
    int n_mat, n_elem;
};

struct KScene {
    DevPrim prims[MAX_PRIMS];
    int n_prims, background;
    real wlo[3], whi[3];
    real eps;         // surface band half-width and smallest root (cm): 8 ulps of the world's FP32 extent
                      // (FP32 tracking) or 1e-6 cm (FP64 tracking, transport.py:155)
};

struct KGrid {
    double* tally;          // [n_slots][nvox] 16-byte scratch cells (kerma, h10) of one batch each
    int tally32;            // cells hold float2 (one vector reduction per visit) instead of double2
    real o[3];
    real h, inv_h;
    int nx, ny, nz;
    long long nvox;
    int enabled;
};

struct KSource {
    int field, rotation, rot_axis, n_angles;
    phys pos[3], dir[3], u[3], v[3];
    phys sid, su, sv, cos_half;
    phys iso[3];
    phys scan;
    int n_e;
    const phys* e;          // energies
    const phys* alias_p;    // alias table
    const int* alias_i;
    // heel effect (source.py:130-149,195-207): heel_n bins along the anode
    // axis; rejection on the relative fluence, then the bin's alias table
    int heel_n, heel_lo, heel_hi;   // bins; first and last bin with fluence
    phys h_u, h_v, span, bin_w;
    const phys* heel_c;      // [heel_n] bin centres
    const phys* heel_f;      // [heel_n] relative fluence
    const int* heel_off;      // [heel_n + 1] each bin's first entry in the tables below
    const phys* heel_e;      // energies
    const phys* heel_q;      // alias probabilities
    const int* heel_a;        // alias entries (table indices)
};

struct KRun {
    long long n;              // histories in this launch
    long long first;          // global index of the first history
    long long batch_size;     // histories per scratch buffer
    int n_scratch;
    int chunk;                // histories a warp takes from the global counter at once
    int fluorescence;
    unsigned long long seed;
    long long max_steps;
    // photon arrays (transport_photons mode)
    double* pos;
    double* dir;
    double* energy;
    int* n_scatter;
    unsigned char* absorbed;
    unsigned char* escaped;
    // reductions
    double* edep;             // [n_scratch][n_mat]
    unsigned long long* counters;   // absorbed, escaped, scatter_sum, n_fluor, steps, voxel visits,
                                    // [6] history counter, [7] segments offered to the queue
    unsigned long long* work;       // global history counter
    unsigned* status;
    struct SegRec* seg;             // track-segment queue of the deferred tally
    long long seg_cap;              // its capacity (records)
    int defer;                      // 1: queue the segments for tally_kernel instead of scoring them
};

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------

__device__ __forceinline__ real fmin3(real a, real b, real c) { return fmin(a, fmin(b, c)); }
__device__ __forceinline__ real fmax3(real a, real b, real c) { return fmax(a, fmax(b, c)); }

// Positions are FP32 (or FP64), so a photon that has just reached a surface sits
// within a few ulps (of the world's largest coordinate) of it on either
// side.  Points inside that band, of half-width tol, are classified by
// their direction: on a surface, a photon is inside the primitive when it
// moves inwards.  The root of the surface the photon sits on is dropped as
// well: a photon grazing a face would otherwise find that face again a
// fraction of an ulp ahead on every step and never leave it.  For planar
// faces (box faces, cylinder caps) the face contributes t = 0; for the
// curved surfaces (sphere, cylinder side) the near root is taken as 0 and
// the far one as the chord -2 b / a of a point on the surface, so a
// photon moving outwards finds no root ahead and one moving inwards finds
// the far side -- the quadratic's own near root, off by rounding of
// order ulp / |radial direction|, can be far above tol at grazing angles.

// Inside the slab |o| <= h, deciding points on a face by the direction d.
__device__ __forceinline__ bool slab_inside(real o, real d, real h, real tol) {
    real a = fabs(o);
    if (a < h - tol) return true;
    if (a > h + tol) return false;
    return o * d <= P(0.0);
}

// Inside the ball |o| <= r (o with n components folded into o2 = |o|^2 and od = o.d).
__device__ __forceinline__ bool ball_inside(real o2, real od, real r, real tol) {
    real lo = fmax(r - tol, (real)0), hi = r + tol;
    if (o2 < lo * lo) return true;
    if (o2 > hi * hi) return false;
    return od <= P(0.0);
}

// Component k of a 3-vector held in registers.  Indexing a register array
// with a runtime k would place the array in local memory for the whole
// kernel, so every runtime axis goes through this select.
template <typename V>
__device__ __forceinline__ V comp(const V v[3], int k) { return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]); }

__device__ __forceinline__ bool contains(const DevPrim& g, const real p[3], const real d[3], real tol) {
    real o0 = p[0] - g.c[0], o1 = p[1] - g.c[1], o2 = p[2] - g.c[2];
    if (g.type == CC_SHAPE_BOX) {
        return slab_inside(o0, d[0], g.h[0], tol) && slab_inside(o1, d[1], g.h[1], tol) &&
               slab_inside(o2, d[2], g.h[2], tol);
    } else if (g.type == CC_SHAPE_SPHERE) {
        return ball_inside(o0 * o0 + o1 * o1 + o2 * o2, o0 * d[0] + o1 * d[1] + o2 * d[2], g.r, tol);
    } else if (g.type == CC_SHAPE_ELLIPSOID) {
        // the unit ball in coordinates scaled by the semi-axes; the band
        // scaled by the smallest semi-axis covers the tol band everywhere
        real u0 = o0 / g.h[0], u1 = o1 / g.h[1], u2 = o2 / g.h[2];
        return ball_inside(u0 * u0 + u1 * u1 + u2 * u2,
                           u0 * d[0] / g.h[0] + u1 * d[1] / g.h[1] + u2 * d[2] / g.h[2], P(1.0), tol * g.r);
    } else {
        const int ax = g.axis;
        const int i0 = ax == 0 ? 1 : 0, i1 = ax == 2 ? 1 : 2;
        real oa = comp(p, i0) - comp(g.c, i0), ob = comp(p, i1) - comp(g.c, i1), ow = comp(p, ax) - comp(g.c, ax);
        return ball_inside(oa * oa + ob * ob, oa * comp(d, i0) + ob * comp(d, i1), g.r, tol) &&
               slab_inside(ow, comp(d, ax), g.hh, tol);
    }
}

__device__ __forceinline__ int locate(const KScene& s, const real p[3], const real d[3]) {
    int m = s.background;
    for (int i = 0; i < s.n_prims; ++i)
        if (contains(s.prims[i], p, d, s.eps)) m = s.prims[i].material;
    return m;
}

// Interval of t where p + t d lies inside the slab [lo, hi] of one axis
// (o = p - c relative coordinate, tol the band of this face); a face the
// point sits on contributes t = 0.  Returns false for a ray parallel to the
// slab outside it.
__device__ __forceinline__ bool slab_pair(real o, real d, real inv, real lo, real hi, real tol,
                                          real& tmin, real& tmax) {
    real dlo = lo - o, dhi = hi - o;
    if (fabs(dlo) <= tol) dlo = P(0.0);
    if (fabs(dhi) <= tol) dhi = P(0.0);
    if (fabs(d) < P(1e-12)) return dlo <= P(0.0) && dhi >= P(0.0);
    real ta = dlo * inv, tb = dhi * inv;
    tmin = fmax(tmin, fmin(ta, tb));
    tmax = fmin(tmax, fmax(ta, tb));
    return true;
}

__device__ __forceinline__ void take_root(real t, real eps, real& best) {
    if (t > eps && t < best) best = t;
}

// Smallest root t > eps of primitive g along the ray (geometry.py:20-99), or best.
__device__ __forceinline__ real prim_next(const DevPrim& g, const real p[3], const real d[3], const real inv[3], real eps,
                           real best) {
    real ox = p[0] - g.c[0], oy = p[1] - g.c[1], oz = p[2] - g.c[2];
    if (g.type == CC_SHAPE_BOX) {
        real tmin = -INFINITY, tmax = INFINITY;
        if (!slab_pair(ox, d[0], inv[0], -g.h[0], g.h[0], eps, tmin, tmax)) return best;
        if (!slab_pair(oy, d[1], inv[1], -g.h[1], g.h[1], eps, tmin, tmax)) return best;
        if (!slab_pair(oz, d[2], inv[2], -g.h[2], g.h[2], eps, tmin, tmax)) return best;
        if (tmin <= tmax) { take_root(tmin, eps, best); take_root(tmax, eps, best); }
        return best;
    } else if (g.type == CC_SHAPE_SPHERE) {
        real b = ox * d[0] + oy * d[1] + oz * d[2];
        real o2 = ox * ox + oy * oy + oz * oz;
        real lo = fmax(g.r - eps, (real)0), hi = g.r + eps;
        if (o2 >= lo * lo && o2 <= hi * hi) {          // on the surface
            if (b <= P(0.0)) take_root(-P(2.0) * b, eps, best);
            return best;
        }
        // squared distance of the line from the centre, computed without cancellation
        real qx = ox - b * d[0], qy = oy - b * d[1], qz = oz - b * d[2];
        real disc = g.r2 - (qx * qx + qy * qy + qz * qz);
        if (disc < P(0.0)) return best;
        real sq = sqrt(disc);
        real c = o2 - g.r2;
        real q = -(b + copysign(sq, b));
        real t1 = q, t2 = (q != P(0.0)) ? c / q : P(0.0);
        take_root(t1, eps, best);
        take_root(t2, eps, best);
        return best;
    } else if (g.type == CC_SHAPE_ELLIPSOID) {
        // |u + t v|^2 = 1 with u = o / h, v = d / h (componentwise)
        real ux = ox / g.h[0], uy = oy / g.h[1], uz = oz / g.h[2];
        real vx = d[0] / g.h[0], vy = d[1] / g.h[1], vz = d[2] / g.h[2];
        real a = vx * vx + vy * vy + vz * vz;
        real b = ux * vx + uy * vy + uz * vz;
        real u2 = ux * ux + uy * uy + uz * uz;
        real tl = eps * g.r;
        real lo = fmax(P(1.0) - tl, (real)0), hi = P(1.0) + tl;
        if (u2 >= lo * lo && u2 <= hi * hi) {            // on the surface
            if (b <= P(0.0)) take_root(-P(2.0) * b / a, eps, best);
            return best;
        }
        real inva = P(1.0) / a;
        real ex = ux - b * inva * vx, ey = uy - b * inva * vy, ez = uz - b * inva * vz;
        real disc = (P(1.0) - (ex * ex + ey * ey + ez * ez)) * a;   // b^2 - a c without cancellation
        if (disc < P(0.0)) return best;
        real q = -(b + copysign(sqrt(disc), b));
        take_root(q * inva, eps, best);
        take_root((q != P(0.0)) ? (u2 - P(1.0)) / q : P(0.0), eps, best);
        return best;
    } else {
        const int ax = g.axis;
        const int i0 = ax == 0 ? 1 : 0, i1 = ax == 2 ? 1 : 2;
        real a0 = comp(p, i0) - comp(g.c, i0), a1 = comp(p, i1) - comp(g.c, i1), aw = comp(p, ax) - comp(g.c, ax);
        real dx = comp(d, i0), dy = comp(d, i1), dw = comp(d, ax);
        real a = dx * dx + dy * dy;
        real rho2 = a0 * a0 + a1 * a1;
        real cc = rho2 - g.r2;
        real tmin, tmax;
        real b = a0 * dx + a1 * dy;
        real lo = fmax(g.r - eps, (real)0), hi = g.r + eps;
        if (rho2 >= lo * lo && rho2 <= hi * hi) {      // on the side surface
            if (b > P(0.0)) return best;
            tmin = P(0.0);
            tmax = a < P(1e-12) ? INFINITY : -P(2.0) * b / a;
        } else if (a < P(1e-12)) {
            if (cc > P(0.0)) return best;        // parallel to the axis, outside the radius
            tmin = -INFINITY; tmax = INFINITY;
        } else {
            real inva = P(1.0) / a;
            real ex = a0 - b * inva * dx, ey = a1 - b * inva * dy;
            real disc = (g.r2 - (ex * ex + ey * ey)) * a;   // b^2 - a c without cancellation
            if (disc < P(0.0)) return best;
            real sq = sqrt(disc);
            real q = -(b + copysign(sq, b));
            real r1 = q * inva, r2 = (q != P(0.0)) ? cc / q : P(0.0);
            tmin = fmin(r1, r2); tmax = fmax(r1, r2);
        }
        if (!slab_pair(aw, dw, comp(inv, ax), -g.hh, g.hh, eps, tmin, tmax)) return best;
        if (tmin <= tmax) { take_root(tmin, eps, best); take_root(tmax, eps, best); }
        return best;
    }
}

// Distance to the world-box exit.
__device__ __forceinline__ real world_exit(const KScene& s, const real p[3], const real d[3],
                                            const real inv[3]) {
    real t = INFINITY;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (d[k] > P(1e-12)) t = fmin(t, (s.whi[k] - p[k]) * inv[k]);
        else if (d[k] < -P(1e-12)) t = fmin(t, (s.wlo[k] - p[k]) * inv[k]);
    }
    return fmax(t, (real)0);
}

// ---------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------

struct Lookup { int idx; phys frac; };

__device__ __forceinline__ Lookup energy_index(const KTables& T, const DevMaterial& m, phys loge) {
    int b = (int)(loge * m.bucket_scale);
    b = max(0, min(N_BUCKETS - 1, b));
    int i = __ldg(T.bucket + m.bucket_off + b);       // last node with log E <= bucket start
    const PNode* x = T.nodes + 2 * (size_t)m.node_off;
    int last = m.n_nodes - 2;
    phys x0 = __ldg(&x[2 * i].x), x1 = __ldg(&x[2 * i + 2].x);
    while (i < last && x1 < loge) {
        ++i;
        x0 = x1;
        x1 = __ldg(&x[2 * i + 2].x);
    }
    Lookup L;
    L.idx = i;
    L.frac = (loge - x0) / (x1 - x0);
    return L;
}

__device__ __forceinline__ phys mu_total(const KTables& T, const DevMaterial& m, const Lookup& L) {
    const PNode* r = T.nodes + 2 * ((size_t)m.node_off + L.idx);
    phys a = __ldg(&r[1].x), b = __ldg(&r[3].x);
    return m.density * p_exp(a + L.frac * (b - a));
}

__device__ __forceinline__ void parts(const KTables& T, const DevMaterial& m, const Lookup& L,
                                      phys& ph, phys& co, phys& ra) {
    const PNode* r = T.nodes + 2 * ((size_t)m.node_off + L.idx);
    PNode a = ldg_node(r), b = ldg_node(r + 2);
    ph = p_exp(a.y + L.frac * (b.y - a.y));
    co = p_exp(a.z + L.frac * (b.z - a.z));
    ra = p_exp(a.w + L.frac * (b.w - a.w));
}

// Element of the material that takes the interaction of kind k (0 photo,
// 1 Compton, 2 Rayleigh), chosen with probability w_i sigma_i / sum
// (physics.py:78-92, 138-152, 223-236).  Returns the element slot.
__device__ __noinline__ int pick_element(const KTables& T, const DevMaterial& m, const Lookup& L, int k, phys r) {
    const int n_el = m.n_el;
    if (n_el == 1) return m.el_slot[0];
    // cumulative sums of w_i sigma_i / sum_j w_j sigma_j, tabulated per node in
    // FP64 on the host and interpolated linearly: first i with r <= cum_i
    const phys* c = T.elem_cum + m.elem_off + (size_t)k * (n_el - 1) * m.n_nodes + L.idx;
    for (int i = 0; i < n_el - 1; ++i) {
        phys c0 = __ldg(c), c1 = __ldg(c + 1);
        if (r <= c0 + L.frac * (c1 - c0)) return m.el_slot[i];
        c += m.n_nodes;
    }
    return m.el_slot[n_el - 1];
}

// Track-length weights at the segment energy: E mu_en (materials.py:310-335,
// transport.py:59-64) and h*(10)/Phi (dose_coefficients.py:32-42), both
// linear in ln E between the material's nodes.
__device__ __forceinline__ void tally_weights(const KTables& T, const DevMaterial& m, const Lookup& L,
                                              phys E, phys& wk, phys& wh) {
    const PNode* r = T.nodes + 2 * ((size_t)m.node_off + L.idx);
    PNode a = ldg_node(r + 1), b = ldg_node(r + 3);
    wk = E * m.density * p_exp(a.y + L.frac * (b.y - a.y));
    wh = p_exp(a.z + L.frac * (b.z - a.z));
}

// ---------------------------------------------------------------------------
// interaction physics
// ---------------------------------------------------------------------------

// S(Z,q)/Z on q = {0} U linspace(1e-3, 20, 1999) (materials.py:484-496), np.interp.
__device__ __forceinline__ phys s_over_z(const phys* s, phys q) {
    const phys q1 = P(1e-3);
    const phys dq = (P(20.0) - P(1e-3)) / P(1998.0);
    if (q <= q1) return __ldg(s + 1) * (q / q1);
    phys u = (q - q1) / dq;
    int j = (int)u;
    if (j >= TABLE_N - 2) return __ldg(s + TABLE_N - 1);
    phys f = u - (phys)j;
    phys a = __ldg(s + 1 + j), b = __ldg(s + 2 + j);
    return a + f * (b - a);
}

// Bound Compton: Kahn-type KN proposal with S(Z,q)/Z rejection (physics.py:41-56, 95-135).
__device__ __forceinline__ void sample_compton(const phys* sz, phys E, HistoryRng& rng, phys& eps_out, phys& cos_out) {
    phys alpha = E / MEC2;
    phys emin = P(1.0) / (P(1.0) + P(2.0) * alpha);
    phys env = P(1.0) / emin + emin;
    phys qscale = E / HC;
    for (int trial = 0; trial < 100000; ++trial) {
        phys x1 = uni(rng), x2 = uni(rng), x3 = uni(rng);
        phys eps = emin + x1 * (P(1.0) - emin);
        phys c = P(1.0) - (P(1.0) / eps - P(1.0)) / alpha;
        phys g = P(1.0) / eps + eps - (P(1.0) - c * c);
        if (x2 * env > g) continue;
        phys cc = fmin(fmax(c, -P(1.0)), P(1.0));
        phys q = qscale * sqrt(P(0.5) * (P(1.0) - cc));
        if (x3 <= s_over_z(sz, q)) { eps_out = eps; cos_out = c; return; }
    }
    eps_out = P(1.0); cos_out = P(1.0);
}

// Rayleigh: inverse of A(x) then (1+cos^2)/2 rejection (physics.py:281-351).
// The row of a target A comes from a uniform-in-A bucket index, then a
// short binary search inside the bucket.
__device__ __forceinline__ bool sample_rayleigh(const phys* rx, const phys* ra, const int* bucket, phys scale,
                                             phys E, HistoryRng& rng, phys& cos_out) {
    phys xmax = (E / HC) * (E / HC);
    if (xmax > __ldg(rx + TABLE_N - 1)) return false;
    // A(x_max): x grid is q^2 with q uniform on [0, 20]
    const phys dq = P(20.0) / (phys)(TABLE_N - 1);
    int j = (int)(sqrt(xmax) / dq);
    j = min(max(j, 0), TABLE_N - 2);
    while (j > 0 && __ldg(rx + j) > xmax) --j;
    while (j < TABLE_N - 2 && __ldg(rx + j + 1) < xmax) ++j;
    phys xa = __ldg(rx + j), xb = __ldg(rx + j + 1);
    phys aa = __ldg(ra + j), ab = __ldg(ra + j + 1);
    phys a_cut = aa + (xmax - xa) / (xb - xa) * (ab - aa);
    for (int trial = 0; trial < 100000; ++trial) {
        phys target = uni(rng) * a_cut;
        int bk = min((int)(target * scale), RAY_BUCKETS - 1);
        int lo = __ldg(bucket + bk), hi = min(__ldg(bucket + bk + 1) + 1, TABLE_N - 1);
        while (hi - lo > 1) {                    // ra[lo] <= target < ra[hi]
            int mid = (lo + hi) >> 1;
            if (__ldg(ra + mid) <= target) lo = mid; else hi = mid;
        }
        phys a0 = __ldg(ra + lo), a1 = __ldg(ra + lo + 1);
        phys x0 = __ldg(rx + lo), x1 = __ldg(rx + lo + 1);
        phys x = (a1 > a0) ? x0 + (target - a0) / (a1 - a0) * (x1 - x0) : x0;
        x = fmin(x, xmax);
        phys c = fmin(fmax(P(1.0) - P(2.0) * x / xmax, -P(1.0)), P(1.0));
        if (uni(rng) <= P(0.5) * (P(1.0) + c * c)) { cos_out = c; return true; }
    }
    cos_out = P(1.0);
    return true;
}

// Photoelectric absorption on a chosen element (physics.py:155-212): above
// the K edge the K shell takes the photon with probability k_prob, it
// relaxes radiatively with probability omega_K and emits one of the K lines
// (cumulative line probabilities), which leaves only when at or above the
// 5 keV cut-off.  Returns the emitted line's energy, 0 when none.
__device__ __forceinline__ phys sample_k_line(const DevElement& el, phys E, int fluorescence, HistoryRng& rng) {
    if (!(fluorescence && el.emits && E > el.k_edge)) return P(0.0);
    const bool is_k = uni(rng) < el.k_prob;
    const bool is_rad = uni(rng) < el.omega;
    if (!(is_k && is_rad)) return P(0.0);
    const phys rl = uni(rng);
    int li = el.n_lines - 1;
    for (int k = 0; k < el.n_lines; ++k) if (rl <= el.line_cum[k]) { li = k; break; }
    return el.line_e[li] >= FLUOR_CUTOFF ? el.line_e[li] : P(0.0);
}

// New direction from cos(theta) and a uniform azimuth (physics.py:354-367).
struct real3 { real x, y, z; };

__device__ __noinline__ real3 scatter_dir(real dx, real dy, real dz, phys cost, phys phi) {
    const real d[3] = {dx, dy, dz};
    real sint = sqrt(fmax((real)0, (real)1 - (real)cost * (real)cost));
    real upx, upy, upz;
    if (fabs(d[2]) < (real)P(0.999)) { upx = 0; upy = 0; upz = 1; } else { upx = 1; upy = 0; upz = 0; }
    real ux = upy * d[2] - upz * d[1], uy = upz * d[0] - upx * d[2], uz = upx * d[1] - upy * d[0];
    real inv = rsqrt_r(ux * ux + uy * uy + uz * uz);
    ux *= inv; uy *= inv; uz *= inv;
    real vx = d[1] * uz - d[2] * uy, vy = d[2] * ux - d[0] * uz, vz = d[0] * uy - d[1] * ux;
    phys sp, cp;
    p_sincos(phi, &sp, &cp);
    real a = sint * cp, b = sint * sp;
    real nx = a * ux + b * vx + cost * d[0];
    real ny = a * uy + b * vy + cost * d[1];
    real nz = a * uz + b * vz + cost * d[2];
    real n = rsqrt_r(nx * nx + ny * ny + nz * nz);
    return real3{nx * n, ny * n, nz * n};
}

__device__ __forceinline__ void scatter_direction(real d[3], phys cost, phys phi) {
    real3 r = scatter_dir(d[0], d[1], d[2], cost, phi);
    d[0] = r.x; d[1] = r.y; d[2] = r.z;
}

__device__ __forceinline__ void isotropic(real d[3], HistoryRng& rng) {
    phys c = P(2.0) * uni(rng) - P(1.0);
    phys s = sqrt(fmax(P(0.0), P(1.0) - c * c));
    phys sp, cp;
    p_sincos(TWO_PI * uni(rng), &sp, &cp);
    d[0] = s * cp; d[1] = s * sp; d[2] = c;
}

// ---------------------------------------------------------------------------
// track-length tally: exact voxel traversal (Amanatides & Woo)
// ---------------------------------------------------------------------------

// One voxel visit: kerma and H*(10) into the batch's scratch, FP64 cells
// (two FP64 reductions).  With FP32 cells switched on for the context, a
// slot that sums at most FP32_SLOT_HISTORIES histories holds FP32 partial
// sums instead, both scored by one 8-byte vector reduction.  Every slot is
// folded into the FP64 totals after its launch.
// The cell kind is a template parameter where the launch knows it, so that
// a kernel holds only the reduction it issues; CELL_RUNTIME reads the grid's
// flag (kernels that serve grids of both kinds).
constexpr int CELL_FP64 = 0, CELL_FP32 = 1, CELL_RUNTIME = 2;

template <int CELL>
__device__ __forceinline__ void score(double* tally, int tally32, int v, real wk_len, real wh_len) {
    if (CELL == CELL_FP32 || (CELL == CELL_RUNTIME && tally32)) {
        asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(reinterpret_cast<float*>(tally + 2 * v)),
                     "f"((float)wk_len), "f"((float)wh_len)
                     : "memory");
    } else {
        atomicAdd(tally + 2 * v, (double)wk_len);
        atomicAdd(tally + 2 * v + 1, (double)wh_len);
    }
}

// Clip the ray p + t d, t in [0, s], to the grid box.  Returns false when
// no part of it lies inside.
__device__ __forceinline__ bool clip_to_grid(const KGrid& G, const real p[3], const real d[3],
                                             const real invd[3], real s, real& t0, real& t1) {
    t0 = P(0.0);
    t1 = s;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        real lo = G.o[k];
        real hi = G.o[k] + G.h * (real)(k == 0 ? G.nx : (k == 1 ? G.ny : G.nz));
        if (fabs(d[k]) < P(1e-12)) {
            if (p[k] < lo || p[k] >= hi) return false;
        } else {
            real ta = (lo - p[k]) * invd[k], tb = (hi - p[k]) * invd[k];
            t0 = fmax(t0, fmin(ta, tb));
            t1 = fmin(t1, fmax(ta, tb));
        }
    }
    return t1 > t0;
}

__device__ __forceinline__ int grid_dim(const KGrid& G, int k) { return k == 0 ? G.nx : (k == 1 ? G.ny : G.nz); }

// Number of voxels the clipped range [t0, t1] crosses (for load balancing).
__device__ __forceinline__ int visit_estimate(const KGrid& G, const real p[3], const real d[3], real t0, real t1) {
    int n = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int nk = grid_dim(G, k);
        int a = max(0, min(nk - 1, (int)floor((p[k] + d[k] * t0 - G.o[k]) * G.inv_h)));
        int b = max(0, min(nk - 1, (int)floor((p[k] + d[k] * t1 - G.o[k]) * G.inv_h)));
        n += abs(b - a);
    }
    return n;
}

// One axis of the traversal: the entry voxel i, the step s (-1, 0, 1), the
// ray parameter tm of the next face crossing and the spacing td of those
// crossings.  A point that rounds onto the far side of a face gets a
// zero-length first cell and steps back in.  Along an axis the ray does
// not move on, the point's side of the neighbouring faces is decided by
// comparing its coordinate with the faces' own: the offset from the grid
// origin keeps only ~1e-7 of the origin's magnitude in FP32, which would
// move the face by up to half an ulp of the grid's extent -- harmless for
// rays that cross faces at random positions, but a beam that runs along a
// face (a pencil beam on a voxel boundary) would have a systematic share of
// its photons scored on the wrong side of it.
__device__ __forceinline__ void walk_axis(real o, real h, real inv_h, int n, real p, real d, real t0, int& i,
                                          int& s, real& tm, real& td) {
    real x = (p + d * t0 - o) * inv_h;
    i = max(0, min(n - 1, (int)floor(x)));
    if (!(fabs(d) > (real)P(1e-12))) {
        if (i > 0 && p < o + (real)i * h) --i;
        else if (i < n - 1 && p >= o + (real)(i + 1) * h) ++i;
    }
    if (d > P(1e-12)) {
        real inv = P(1.0) / d;
        s = 1;
        tm = (o + (real)(i + 1) * h - p) * inv;
        td = h * inv;
    } else if (d < -P(1e-12)) {
        real inv = P(1.0) / d;
        s = -1;
        tm = (o + (real)i * h - p) * inv;
        td = -h * inv;
    } else {
        s = 0;
        tm = INFINITY;
        td = INFINITY;
    }
}

// Exact voxel traversal (Amanatides & Woo) of p + t d over [t0, t1], which
// lies inside the grid box; scores weight x overlap length per voxel.  The
// per-axis state is held in scalars and the crossing axis picked by
// selects: a register array indexed by the crossing axis would live in
// local memory.
template <int CELL = CELL_RUNTIME>
__device__ __forceinline__ int walk_range(const KGrid& G, double* tally, const real p[3], const real d[3],
                                          real t0, real t1, phys wk, phys wh) {
    int ix, iy, iz, sx, sy, sz;
    real mx, my, mz, dx, dy, dz;
    walk_axis(G.o[0], G.h, G.inv_h, G.nx, p[0], d[0], t0, ix, sx, mx, dx);
    walk_axis(G.o[1], G.h, G.inv_h, G.ny, p[1], d[1], t0, iy, sy, my, dy);
    walk_axis(G.o[2], G.h, G.inv_h, G.nz, p[2], d[2], t0, iz, sz, mz, dz);
    real t = t0;
    int guard = G.nx + G.ny + G.nz + 4;
    int visits = 0;
    // flat index (C order, tally.py:292) updated incrementally; grids are < 2^31 voxels
    const int vx = sx * G.ny * G.nz, vy = sy * G.nz, vz = sz;
    int v = (ix * G.ny + iy) * G.nz + iz;
    while (t < t1 && guard-- > 0) {
        // the axis whose face comes first; ties go to the later axis, except
        // that x beats z only when strictly first
        const bool ax0 = (mx < my) && (mx < mz);
        const bool ax1 = !(mx < my) && (my < mz);
        const bool ax2 = !ax0 && !ax1;
        real tn = fmin(ax0 ? mx : (ax1 ? my : mz), t1);
        real len = tn - t;
        if (len > P(0.0)) {
            score<CELL>(tally, G.tally32, v, wk * len, wh * len);
            ++visits;
        }
        t = tn;
        if (t >= t1) break;
        ix += ax0 ? sx : 0;
        iy += ax1 ? sy : 0;
        iz += ax2 ? sz : 0;
        if ((unsigned)ix >= (unsigned)G.nx || (unsigned)iy >= (unsigned)G.ny || (unsigned)iz >= (unsigned)G.nz) break;
        v += ax0 ? vx : (ax1 ? vy : vz);
        if (ax0) mx += dx;
        if (ax1) my += dy;
        if (ax2) mz += dz;
    }
    return visits;
}

// One track segment to score: the warp's segments in shared memory, and the
// records of the deferred tally's queue in HBM.
struct SegRec {
    real p[3], d[3];
    real t0, t1;
    phys wk, wh;
    int batch, m;           // scratch slot; pieces of at most TALLY_PIECE visits
};

// ---------------------------------------------------------------------------
// source (source.py:67-210)
// ---------------------------------------------------------------------------

__device__ __forceinline__ void rotate(phys v[3], int axis, phys ca, phys sa) {
    // Rodrigues rotation about a coordinate axis
    phys a0 = v[0], a1 = v[1], a2 = v[2];
    if (axis == 0) { v[1] = a1 * ca - a2 * sa; v[2] = a1 * sa + a2 * ca; }
    else if (axis == 1) { v[0] = a0 * ca + a2 * sa; v[2] = -a0 * sa + a2 * ca; }
    else { v[0] = a0 * ca - a1 * sa; v[1] = a0 * sa + a1 * ca; }
}

// np.interp(s, centres, fluence): clamped to the end values outside.
__device__ __forceinline__ phys heel_fluence(const KSource& S, phys s) {
    const int n = S.heel_n;
    if (s <= __ldg(S.heel_c)) return __ldg(S.heel_f);
    if (s >= __ldg(S.heel_c + n - 1)) return __ldg(S.heel_f + n - 1);
    int lo = 0, hi = n - 1;                  // c[lo] < s < c[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(S.heel_c + mid) <= s) lo = mid; else hi = mid;
    }
    const phys c0 = __ldg(S.heel_c + lo), c1 = __ldg(S.heel_c + hi);
    const phys f0 = __ldg(S.heel_f + lo), f1 = __ldg(S.heel_f + hi);
    return f0 + (s - c0) / (c1 - c0) * (f1 - f0);
}

// Energy of a photon at heel coordinate s: the alias table of its bin,
// clamped to the bins that have fluence (source.py:195-207).
__device__ __forceinline__ phys heel_energy(const KSource& S, phys s, HistoryRng& rng) {
    int b = (int)((s + S.span) / S.bin_w);
    b = min(max(b, 0), S.heel_n - 1);
    b = min(max(b, S.heel_lo), S.heel_hi);
    const int off = __ldg(S.heel_off + b), nb = __ldg(S.heel_off + b + 1) - off;
    const phys r = uni(rng) * (phys)nb;
    const int i = min((int)r, nb - 1);
    const int pick = (r - (phys)i <= __ldg(S.heel_q + off + i)) ? off + i : __ldg(S.heel_a + off + i);
    return __ldg(S.heel_e + pick);
}

constexpr int HEEL_MAX_TRIALS = 100000;

// HEEL: the source may carry the heel effect (a separate instantiation, so
// that the kernels of sources without it keep their registers).
template <bool HEEL>
__device__ __forceinline__ void sample_source(const KSource& S, HistoryRng& rng, real p[3], real d[3], phys& E) {
    phys pos[3] = {S.pos[0], S.pos[1], S.pos[2]};
    phys dir[3] = {S.dir[0], S.dir[1], S.dir[2]};
    phys u[3] = {S.u[0], S.u[1], S.u[2]};
    phys v[3] = {S.v[0], S.v[1], S.v[2]};
    if (S.rotation) {
        phys ang;
        if (S.n_angles > 0) {
            uint32_t k = (uint32_t)(((uint64_t)rng.next_u32() * (uint64_t)S.n_angles) >> 32);
            ang = TWO_PI * (phys)k / (phys)S.n_angles;
        } else {
            ang = TWO_PI * (uni(rng) - P(0.5)) + P(3.14159265358979);
        }
        phys sa, ca;
        p_sincos(ang, &sa, &ca);
        phys rel[3] = {pos[0] - S.iso[0], pos[1] - S.iso[1], pos[2] - S.iso[2]};
        rotate(rel, S.rot_axis, ca, sa);
        rotate(dir, S.rot_axis, ca, sa);
        rotate(u, S.rot_axis, ca, sa);
        rotate(v, S.rot_axis, ca, sa);
        pos[0] = S.iso[0] + rel[0]; pos[1] = S.iso[1] + rel[1]; pos[2] = S.iso[2] + rel[2];
        if (S.scan > P(0.0)) {
            phys shift = S.scan * (uni(rng) - P(0.5));
            pos[0] += S.rot_axis == 0 ? shift : P(0.0);
            pos[1] += S.rot_axis == 1 ? shift : P(0.0);
            pos[2] += S.rot_axis == 2 ? shift : P(0.0);
        }
    }
    const bool heel = HEEL && S.heel_n > 0 && S.field != CC_FIELD_PARALLEL;
    phys s_heel = P(0.0);
    if (S.field == CC_FIELD_CONE) {
        phys c, sp, cp;
        for (int trial = 0; ; ++trial) {
            c = S.cos_half + (P(1.0) - S.cos_half) * (P(1.0) - uni(rng));
            p_sincos(TWO_PI * uni(rng), &sp, &cp);
            if (!heel) break;
            // the direction's offset along the heel axis on the SID plane
            s_heel = S.sid * (sqrt(fmax(P(0.0), P(1.0) - c * c)) / c) * (cp * S.h_u + sp * S.h_v);
            if (uni(rng) < heel_fluence(S, s_heel) || trial >= HEEL_MAX_TRIALS) break;
        }
        phys s = sqrt(fmax(P(0.0), P(1.0) - c * c));
        for (int k = 0; k < 3; ++k) { p[k] = pos[k]; d[k] = c * dir[k] + s * cp * u[k] + s * sp * v[k]; }
    } else if (S.field == CC_FIELD_PARALLEL) {
        phys a = S.su * (uni(rng) - P(0.5)), b = S.sv * (uni(rng) - P(0.5));
        for (int k = 0; k < 3; ++k) { p[k] = pos[k] + a * u[k] + b * v[k]; d[k] = dir[k]; }
    } else {
        phys a, b;
        for (int trial = 0; ; ++trial) {
            a = S.su * (uni(rng) - P(0.5));
            b = S.sv * (uni(rng) - P(0.5));
            if (!heel) break;
            s_heel = a * S.h_u + b * S.h_v;
            if (uni(rng) < heel_fluence(S, s_heel) || trial >= HEEL_MAX_TRIALS) break;
        }
        phys t[3];
        for (int k = 0; k < 3; ++k) t[k] = dir[k] * S.sid + a * u[k] + b * v[k];
        phys inv = rsqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        for (int k = 0; k < 3; ++k) { p[k] = pos[k]; d[k] = t[k] * inv; }
    }
    if (heel) {
        E = heel_energy(S, s_heel, rng);
        return;
    }
    // discrete spectrum by Walker's alias method
    phys r = uni(rng) * (phys)S.n_e;
    int i = min((int)r, S.n_e - 1);
    phys f = r - (phys)i;
    int pick = (f <= __ldg(S.alias_p + i)) ? i : __ldg(S.alias_i + i);
    E = __ldg(S.e + pick);
}

// ---------------------------------------------------------------------------
// the transport kernel
// ---------------------------------------------------------------------------

// Histories a warp takes from the global counter at once.  The histories in
// flight span warps x chunk indices, i.e. several batches, and every batch
// scores into its own scratch slot.  A small grid (a slot of a few MB) wants
// that spread: the hot voxels then have several copies in L2 and their
// atomics contend less.  A grid whose slot is near the L2 size wants the
// opposite, fewer slots in flight, or its atomics miss in L2.  Measured on
// the room workload (6 MB slots) 32 histories per chunk were 1.9x slower than
// 256, on the CT workload (246 MB slots) 9 % faster.
constexpr int HIST_CHUNK_SPREAD = 256;
constexpr int HIST_CHUNK_COMPACT = 32;
constexpr size_t SLOT_BYTES_COMPACT = (size_t)32 << 20;     // slots above this use the compact chunk
// Voxel visits per piece when a warp splits its track segments.  The split
// of a segment depends on that segment alone, never on the warp's other
// lanes, so every piece -- and every length it scores -- is the same
// whichever histories share a warp; runs with one seed then differ only in
// the order of the FP64 additions.
#ifndef TALLY_PIECE
#define TALLY_PIECE 16
#endif
constexpr int BLOCK = 256;
constexpr int WARPS_PER_BLOCK = BLOCK / 32;
// A thread's 32-bit counters go to the block's 64-bit ones once any reaches
// 2^30: one history adds far less than the remaining 2^31 (its steps are
// capped by the step limit, its voxel visits by the grid's size per step).
constexpr unsigned COUNTER_FLUSH = 1u << 30;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int warp_inclusive_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Piece k of m of the segment [t0, t1]: equal-length cuts that depend on the
// segment alone.
__device__ __forceinline__ void piece_range(real t0, real t1, int m, int k, real& ta, real& tz) {
    const real dt = (t1 - t0) / (real)m;
    ta = t0 + dt * (real)k;
    tz = (k == m - 1) ? t1 : ta + dt;
}

// The warp scores its segments together: lane l's segment (if m > 0) is in
// seg[l]; every segment is cut into m pieces and the lanes walk all pieces
// round-robin, so every lane walks about the same number of voxels.
template <int CELL = CELL_RUNTIME>
__device__ __forceinline__ void score_warp_segments(const KGrid& G, const SegRec* seg, int* pre, int lane, int m,
                                                    unsigned& c_vox) {
    int incl = warp_inclusive_scan(m, lane);
    pre[lane] = incl - m;
    if (lane == 31) pre[32] = incl;
    __syncwarp();
    const int U = pre[32];
    for (int u = lane; u < U; u += 32) {
        int lo = 0, hi = 32;            // pre[lo] <= u < pre[hi]
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (pre[mid] <= u) lo = mid; else hi = mid;
        }
        const SegRec& q = seg[lo];
        const int k = u - pre[lo];
        real ta, tz;
        piece_range(q.t0, q.t1, q.m, k, ta, tz);
        int nv = walk_range<CELL>(G, G.tally + (size_t)q.batch * 2 * G.nvox, q.p, q.d, ta, tz, q.wk, q.wh);
        c_vox += max(nv - (k > 0 ? 1 : 0), 0);   // a cut voxel is one visit
    }
    __syncwarp();
}

// Deferred tally (a context option, off by default): the transport kernel
// appends its in-grid segments to a queue in HBM, and tally_kernel scores
// them with full warps at its own occupancy.  Scores are the same pieces as
// the inline tally's.  Measured slower on B200 (room 3.69e8 vs 5.24e8,
// CT 1.79e8 vs 2.46e8 histories/s): the tally is bound by its FP64 atomics,
// which the inline tally overlaps with other warps' transport arithmetic.

// Each loop iteration is one transport step of every lane, in three
// warp-synchronous phases:
//   1. lanes without a photon start the next history; every lane finds its
//      material, mu and next boundary and decides its segment;
//   2. the warp scores all its segments together: long segments are cut
//      into equal-length pieces of at most TALLY_PIECE voxel visits, and the
//      lanes walk the pieces round-robin, so every lane walks about the same
//      number of voxels;
//   3. lanes move their photon and sample the interaction, if any.
// Four 256-thread blocks per SM: the register budget (<= 64) that this asks
// for costs no spills and hides more latency than two or three blocks.
#ifndef CC_MIN_BLOCKS
#define CC_MIN_BLOCKS 4
#endif

// The tally variant TV of a launch: CELL_FP64 or CELL_FP32 scores inline
// with that one reduction; TV_DEFER queues the segments (the fallback walk
// reads the grid's cell flag).  Each instantiation holds one copy of the
// voxel walk, which keeps the loop's code small.
constexpr int TV_DEFER = 3;

template <bool FROM_SOURCE, bool TALLY, bool HEEL = false, int TV = CELL_FP64>
__global__ void __launch_bounds__(BLOCK, CC_MIN_BLOCKS)
transport_kernel(const KTables T, const KScene S, const KGrid G, const KSource SRC, const KRun R) {
    extern __shared__ double s_edep[];             // [n_scratch][n_mat]
    __shared__ unsigned long long s_cnt[6];
    __shared__ SegRec s_seg[TALLY ? WARPS_PER_BLOCK : 1][32];
    __shared__ int s_pre[TALLY ? WARPS_PER_BLOCK : 1][33];
    const int n_acc = R.n_scratch * T.n_mat;
    for (int i = threadIdx.x; i < n_acc; i += blockDim.x) s_edep[i] = 0.0;
    if (threadIdx.x < 6) s_cnt[threadIdx.x] = 0ull;
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // per-thread counters in 32 bits (registers are the kernel's limit); a
    // thread hands them to the block's 64-bit counters before they near 2^31
    unsigned c_abs = 0, c_esc = 0, c_sc = 0, c_fl = 0, c_steps = 0, c_vox = 0;

    // a launch that leaves the chunk unset takes the spread default (a zero
    // chunk would never advance the counter)
    const int chunk = R.chunk > 0 ? R.chunk : HIST_CHUNK_SPREAD;
    // warp-local pool [pool_next, pool_end)
    long long pool_next = 0, pool_end = 0;
    bool live = false;
    long long h = 0;
    real p[3], d[3];
    phys E = P(0.), tau = P(0.);
    int nsc = 0, mat = -1, batch = 0;
    int steps = 0;
    HistoryRng rng;

    while (true) {
        // ---- phase 1a: regeneration ----
        unsigned need = __ballot_sync(FULL, !live);
        while (need) {
            if (pool_next >= pool_end) {
                long long base = 0;
                if (lane == 0) base = (long long)atomicAdd(R.work, (unsigned long long)chunk);
                base = __shfl_sync(FULL, base, 0);
                if (base >= R.n) break;
                pool_next = base;
                pool_end = min(base + chunk, R.n);
            }
            int rank = __popc(need & ((1u << lane) - 1u));
            long long avail = pool_end - pool_next;
            int take = (int)min((long long)__popc(need), avail);
            if (!live && rank < take) {
                h = pool_next + rank;
                live = true;
                long long gh = R.first + h;
                rng.init(R.seed, (unsigned long long)gh, 0u);
                batch = (int)(h / R.batch_size);
                if (batch >= R.n_scratch) batch = R.n_scratch - 1;
                if (FROM_SOURCE) {
                    sample_source<HEEL>(SRC, rng, p, d, E);
                } else {
                    for (int k = 0; k < 3; ++k) {
                        p[k] = (real)R.pos[3 * h + k];
                        d[k] = (real)R.dir[3 * h + k];
                    }
                    E = (phys)R.energy[h];
                }
                tau = -p_log(uni(rng));
                nsc = 0;
                mat = -1;
                steps = 0;
            }
            pool_next += take;
            need = __ballot_sync(FULL, !live);
        }
        if (__all_sync(FULL, !live)) break;

        // ---- phase 1b: material, mu, next boundary ----
        bool go = live;
        bool interact = false, escape = false;
        real s = 0, t0 = 0, t1 = 0;
        phys tau_b = P(0.), loge = P(0.), wk = P(0.), wh = P(0.);
        int tal_n = 0;
        Lookup L;
        L.idx = 0;
        L.frac = P(0.);
        if (go) {
            ++steps;
            if (mat < 0) mat = locate(S, p, d);
            if (mat >= T.n_mat) {
                atomicOr(R.status, ST_BOUNDS);
                go = live = false;
            } else if (!(E >= E_MIN_KEV && E <= E_MAX_KEV)) {
                atomicOr(R.status, ST_ENERGY);
                go = live = false;
            }
        }
        if (go) {
            const DevMaterial& M = T.mats[mat];
            loge = p_log(E);
            L = energy_index(T, M, loge);
            phys mu = mu_total(T, M, L);
            const real invd[3] = {(real)1 / d[0], (real)1 / d[1], (real)1 / d[2]};
            real tb = INFINITY;
            for (int i = 0; i < S.n_prims; ++i) tb = prim_next(S.prims[i], p, d, invd, S.eps, tb);
            real tw = world_exit(S, p, d, invd);
            escape = tw <= tb;
            tb = fmin(tb, tw);
            tau_b = (phys)(mu * tb);
            interact = tau < tau_b;
            s = interact ? (real)tau / (real)fmax(mu, P(1e-30)) : tb;
            if (TALLY && clip_to_grid(G, p, d, invd, s, t0, t1)) {
                tally_weights(T, M, L, E, wk, wh);
                tal_n = visit_estimate(G, p, d, t0, t1);
            }
        }

        // ---- phase 2: the warp scores its segments, or queues them ----
        if (TALLY && TV == TV_DEFER) {
            const bool has = tal_n > 0;
            const unsigned mask = __ballot_sync(FULL, has);
            if (mask) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(R.counters + 7, (unsigned long long)__popc(mask));
                base = __shfl_sync(FULL, base, 0);
                if (has) {
                    const int m = (tal_n + TALLY_PIECE - 1) / TALLY_PIECE;
                    const unsigned long long idx = base + __popc(mask & ((1u << lane) - 1u));
                    if (idx < (unsigned long long)R.seg_cap) {
                        SegRec& r = R.seg[idx];
                        r.p[0] = p[0]; r.p[1] = p[1]; r.p[2] = p[2];
                        r.d[0] = d[0]; r.d[1] = d[1]; r.d[2] = d[2];
                        r.t0 = t0; r.t1 = t1; r.wk = wk; r.wh = wh; r.batch = batch; r.m = m;
                    } else {
                        // queue full: this lane walks the same pieces itself
                        for (int k = 0; k < m; ++k) {
                            real ta, tz;
                            piece_range(t0, t1, m, k, ta, tz);
                            int nv = walk_range(G, G.tally + (size_t)batch * 2 * G.nvox, p, d, ta, tz, wk, wh);
                            c_vox += max(nv - (k > 0 ? 1 : 0), 0);
                        }
                    }
                }
            }
        } else if (TALLY) {
            if (__any_sync(FULL, tal_n > 0)) {
                int m = (tal_n + TALLY_PIECE - 1) / TALLY_PIECE;
                if (m > 0) {
                    SegRec& r = s_seg[warp][lane];
                    r.p[0] = p[0]; r.p[1] = p[1]; r.p[2] = p[2];
                    r.d[0] = d[0]; r.d[1] = d[1]; r.d[2] = d[2];
                    r.t0 = t0; r.t1 = t1; r.wk = wk; r.wh = wh; r.batch = batch; r.m = m;
                }
                score_warp_segments<TV == TV_DEFER ? CELL_RUNTIME : TV>(G, s_seg[warp], s_pre[warp], lane, m, c_vox);
            }
        }
        if (TALLY && c_vox >= COUNTER_FLUSH) {
            atomicAdd(&s_cnt[5], (unsigned long long)c_vox);
            c_vox = 0;
        }
        if (!go) continue;

        // ---- phase 3: move, cross or interact ----
        const DevMaterial& M = T.mats[mat];
        p[0] += d[0] * s; p[1] += d[1] * s; p[2] += d[2] * s;
        bool done = false;
        bool esc = false, absd = false;
        if (!interact) {
            tau -= tau_b;
            if (escape) { esc = true; done = true; }
            mat = -1;                      // re-locate after the crossing
        } else {
            phys ph, co, ra;
            parts(T, M, L, ph, co, ra);
            phys tot = ph + co + ra;
            phys r = uni(rng) * tot;
            ++nsc;
            const int kind = r < ph ? 0 : (r < ph + co ? 1 : 2);
            // The element draw, the new direction and the new free path are
            // common to the three interactions; they run outside the branches
            // so that every interacting lane of the warp executes them together.
            const int slot = pick_element(T, M, L, kind, uni(rng));
            phys cost = P(1.0), e_new = E, dep = P(0.0);
            if (kind == 0) {
                // photoelectric, K fluorescence (physics.py:155-212, transport.py:174-198)
                const phys e_line = sample_k_line(T.elems[slot], E, R.fluorescence, rng);
                const bool emit = e_line > P(0.0);
                dep = emit ? E - e_line : E;
                if (emit) {
                    ++c_fl;
                    e_new = e_line;
                } else {
                    absd = true;
                    done = true;
                }
            } else if (kind == 1) {
                phys eps;
                sample_compton(T.sq + (size_t)slot * TABLE_N, E, rng, eps, cost);
                e_new = E * eps;
                dep = E - e_new;
            } else if (!sample_rayleigh(T.rx + (size_t)slot * TABLE_N, T.ra + (size_t)slot * TABLE_N,
                                        T.ray_bucket + (size_t)slot * (RAY_BUCKETS + 1), T.elems[slot].ray_scale,
                                        E, rng, cost)) {
                atomicOr(R.status, ST_RAYLEIGH_Q);
                live = false;
                continue;
            }
            if (kind < 2) atomicAdd(&s_edep[batch * T.n_mat + mat], (double)dep);
            if (!done) {
                if (kind == 0) isotropic(d, rng);                     // the fluorescence photon
                else scatter_direction(d, cost, TWO_PI * uni(rng));
                E = e_new;
                tau = -p_log(uni(rng));
            }
            mat = -1;                      // new direction: re-locate (material_at every round)
        }
        if (!done && steps >= R.max_steps) {
            atomicOr(R.status, ST_STEPS);
            done = true;
        }
        if (done) {
            c_steps += (unsigned)steps;
            c_sc += nsc;
            if (esc) ++c_esc;
            if (absd) ++c_abs;
            if ((c_steps | c_vox | c_sc) >= COUNTER_FLUSH) {
                atomicAdd(&s_cnt[0], (unsigned long long)c_abs);
                atomicAdd(&s_cnt[1], (unsigned long long)c_esc);
                atomicAdd(&s_cnt[2], (unsigned long long)c_sc);
                atomicAdd(&s_cnt[3], (unsigned long long)c_fl);
                atomicAdd(&s_cnt[4], (unsigned long long)c_steps);
                atomicAdd(&s_cnt[5], (unsigned long long)c_vox);
                c_abs = c_esc = c_sc = c_fl = c_steps = c_vox = 0;
            }
            if (!FROM_SOURCE) {
                for (int k = 0; k < 3; ++k) {
                    R.pos[3 * h + k] = (double)p[k] + (esc ? (double)d[k] * 1e-6 : 0.0);
                    R.dir[3 * h + k] = (double)d[k];
                }
                R.energy[h] = (double)E;
                if (R.n_scatter) R.n_scatter[h] = nsc;
                if (R.absorbed) R.absorbed[h] = absd ? 1 : 0;
                if (R.escaped) R.escaped[h] = esc ? 1 : 0;
            }
            live = false;
        }
    }
    // ---- reductions ----
    atomicAdd(&s_cnt[0], (unsigned long long)c_abs);
    atomicAdd(&s_cnt[1], (unsigned long long)c_esc);
    atomicAdd(&s_cnt[2], (unsigned long long)c_sc);
    atomicAdd(&s_cnt[3], (unsigned long long)c_fl);
    atomicAdd(&s_cnt[4], (unsigned long long)c_steps);
    atomicAdd(&s_cnt[5], (unsigned long long)c_vox);
    __syncthreads();
    for (int i = threadIdx.x; i < n_acc; i += blockDim.x)
        if (s_edep[i] != 0.0) atomicAdd(R.edep + i, s_edep[i]);
    if (threadIdx.x < 6) atomicAdd(R.counters + threadIdx.x, s_cnt[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// deferred tally: the queued segments of one launch
// ---------------------------------------------------------------------------

constexpr int TALLY_MIN_BLOCKS = 6;
constexpr size_t SEG_QUEUE_MAX_BYTES = (size_t)6 << 30;   // beyond it, lanes walk their own segments

__global__ void __launch_bounds__(BLOCK, TALLY_MIN_BLOCKS)
tally_kernel(const KGrid G, const SegRec* __restrict__ seg, const unsigned long long* __restrict__ offered,
             long long cap, unsigned long long* __restrict__ counters) {
    __shared__ SegRec s_seg[WARPS_PER_BLOCK][32];
    __shared__ int s_pre[WARPS_PER_BLOCK][33];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long n = min((long long)*offered, cap);      // offers beyond the capacity were walked in place
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned c_vox = 0;
    unsigned long long c_tot = 0;
    for (long long b = gw * 32; b < n; b += nw * 32) {       // warp-uniform bounds
        const long long i = b + lane;
        int m = 0;
        if (i < n) {
            s_seg[warp][lane] = seg[i];
            m = s_seg[warp][lane].m;
        }
        score_warp_segments(G, s_seg[warp], s_pre[warp], lane, m, c_vox);
        if (c_vox >= COUNTER_FLUSH) { c_tot += c_vox; c_vox = 0; }
    }
    c_tot += c_vox;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c_tot += __shfl_xor_sync(FULL, c_tot, o);
    if (lane == 0 && c_tot) atomicAdd(counters + 5, c_tot);
}

// ---------------------------------------------------------------------------
// batched multi-scene transport (one launch over many scenes)
// ---------------------------------------------------------------------------

struct KBatch {
    const KScene* scenes;           // [n_scenes]
    const KSource* sources;         // [n_scenes]
    const KGrid* grids;             // [n_scenes] (tally pointers at the first scratch slot)
    const long long* chunk_first;   // [n_scenes + 1] first chunk of each scene
    const long long* n_hist;        // [n_scenes]
    unsigned long long* scene_cnt;  // [n_scenes][4] absorbed, escaped, scatter_sum, fluorescence
    const unsigned long long* run;  // [2] seed, fluorescence (written before each replay)
    int n_scenes;
    int chunk;                      // histories per chunk (a chunk never spans two scenes)
    int slots;                      // batch-statistics slots per scene (1 = totals only)
    long long n_chunks;
};

static_assert(sizeof(KSource) % 8 == 0 && sizeof(KGrid) % 8 == 0, "device tables hold 8-byte fields");

struct SegRecB {
    real p[3], d[3];
    real t0, t1;
    phys wk, wh;
    int scene, slot, m;
};

__device__ __forceinline__ int scene_of_chunk(const KBatch& B, long long c) {
    int lo = 0, hi = B.n_scenes;            // chunk_first[lo] <= c < chunk_first[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(B.chunk_first + mid) <= c) lo = mid; else hi = mid;
    }
    return lo;
}

// Per-scene outcome counts, summed over the lanes of the warp that end a
// history in this iteration with the same scene.
__device__ __forceinline__ void add_scene_counts(const KBatch& B, bool ended, int sc, unsigned a, unsigned e,
                                                 unsigned nsc, unsigned fl, int lane) {
    unsigned enders = __ballot_sync(FULL, ended);
    if (!ended) return;
    unsigned grp = __match_any_sync(enders, sc);
    int leader = __ffs(grp) - 1;
    unsigned va = a, ve = e, vs = nsc, vf = fl;
    // sum over the group with shuffles of the group members
    unsigned sa = 0, se = 0, ss = 0, sf = 0;
    for (unsigned m = grp; m; m &= m - 1) {
        int src = __ffs(m) - 1;
        sa += __shfl_sync(grp, va, src);
        se += __shfl_sync(grp, ve, src);
        ss += __shfl_sync(grp, vs, src);
        sf += __shfl_sync(grp, vf, src);
    }
    if (lane == leader) {
        unsigned long long* c = B.scene_cnt + 4 * (size_t)sc;
        if (sa) atomicAdd(c + 0, (unsigned long long)sa);
        if (se) atomicAdd(c + 1, (unsigned long long)se);
        if (ss) atomicAdd(c + 2, (unsigned long long)ss);
        if (sf) atomicAdd(c + 3, (unsigned long long)sf);
    }
}

template <bool TALLY, bool HEEL = false>
__global__ void __launch_bounds__(BLOCK, CC_MIN_BLOCKS)
batch_kernel(const KTables T, const KBatch B, const KRun R) {
    __shared__ SegRecB s_seg[TALLY ? WARPS_PER_BLOCK : 1][32];
    __shared__ int s_pre[TALLY ? WARPS_PER_BLOCK : 1][33];
    __shared__ unsigned long long s_cnt[2];
    if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0ull;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const unsigned long long seed = __ldg(B.run);
    const int fluorescence = (int)__ldg(B.run + 1);
    unsigned c_steps = 0, c_vox = 0;            // 32-bit, handed on before they near 2^31

    long long pool_next = 0, pool_end = 0;
    int pool_scene = 0;
    bool live = false;
    int sc = 0, slot = 0;
    long long li = 0;
    real p[3], d[3];
    phys E = P(0.), tau = P(0.);
    int nsc = 0, mat = -1;
    int steps = 0;
    HistoryRng rng;

    while (true) {
        // ---- regeneration ----
        unsigned need = __ballot_sync(FULL, !live);
        while (need) {
            if (pool_next >= pool_end) {
                long long c = 0;
                if (lane == 0) c = (long long)atomicAdd(R.work, 1ull);
                c = __shfl_sync(FULL, c, 0);
                if (c >= B.n_chunks) break;
                pool_scene = scene_of_chunk(B, c);
                long long nh = __ldg(B.n_hist + pool_scene);
                pool_next = (c - __ldg(B.chunk_first + pool_scene)) * (long long)B.chunk;
                pool_end = min(pool_next + (long long)B.chunk, nh);
            }
            int rank = __popc(need & ((1u << lane) - 1u));
            long long avail = pool_end - pool_next;
            int take = (int)min((long long)__popc(need), avail);
            if (!live && rank < take) {
                li = pool_next + rank;
                sc = pool_scene;
                live = true;
                rng.init(seed, ((unsigned long long)sc << 40) + (unsigned long long)li, 0u);
                long long nh = __ldg(B.n_hist + sc);
                slot = (int)((li * B.slots) / nh);
                sample_source<HEEL>(B.sources[sc], rng, p, d, E);
                tau = -p_log(uni(rng));
                nsc = 0;
                mat = -1;
                steps = 0;
            }
            pool_next += take;
            need = __ballot_sync(FULL, !live);
        }
        if (__all_sync(FULL, !live)) break;

        // ---- phase 1 ----
        const KScene& S = B.scenes[sc];
        bool go = live;
        bool interact = false, escape = false;
        real s = 0, t0 = 0, t1 = 0;
        phys tau_b = P(0.), loge = P(0.), wk = P(0.), wh = P(0.);
        int tal_n = 0;
        Lookup L;
        L.idx = 0;
        L.frac = P(0.);
        if (go) {
            ++steps;
            if (mat < 0) mat = locate(S, p, d);
            if (mat >= T.n_mat) {
                atomicOr(R.status, ST_BOUNDS);
                go = live = false;
            } else if (!(E >= E_MIN_KEV && E <= E_MAX_KEV)) {
                atomicOr(R.status, ST_ENERGY);
                go = live = false;
            }
        }
        if (go) {
            const DevMaterial& M = T.mats[mat];
            loge = p_log(E);
            L = energy_index(T, M, loge);
            phys mu = mu_total(T, M, L);
            const real invd[3] = {(real)1 / d[0], (real)1 / d[1], (real)1 / d[2]};
            real tb = INFINITY;
            const int np = S.n_prims;
            for (int i = 0; i < np; ++i) tb = prim_next(S.prims[i], p, d, invd, S.eps, tb);
            real tw = world_exit(S, p, d, invd);
            escape = tw <= tb;
            tb = fmin(tb, tw);
            tau_b = (phys)(mu * tb);
            interact = tau < tau_b;
            s = interact ? (real)tau / (real)fmax(mu, P(1e-30)) : tb;
            if (TALLY && clip_to_grid(B.grids[sc], p, d, invd, s, t0, t1)) {
                tally_weights(T, M, L, E, wk, wh);
                tal_n = visit_estimate(B.grids[sc], p, d, t0, t1);
            }
        }

        // ---- phase 2: the warp scores its segments together ----
        if (TALLY) {
            if (__any_sync(FULL, tal_n > 0)) {
                int m = (tal_n + TALLY_PIECE - 1) / TALLY_PIECE;
                if (m > 0) {
                    SegRecB& r = s_seg[warp][lane];
                    r.p[0] = p[0]; r.p[1] = p[1]; r.p[2] = p[2];
                    r.d[0] = d[0]; r.d[1] = d[1]; r.d[2] = d[2];
                    r.t0 = t0; r.t1 = t1; r.wk = wk; r.wh = wh; r.scene = sc; r.slot = slot; r.m = m;
                }
                int incl = warp_inclusive_scan(m, lane);
                s_pre[warp][lane] = incl - m;
                if (lane == 31) s_pre[warp][32] = incl;
                __syncwarp();
                const int U = s_pre[warp][32];
                for (int u = lane; u < U; u += 32) {
                    int lo = 0, hi = 32;
                    while (hi - lo > 1) {
                        int mid = (lo + hi) >> 1;
                        if (s_pre[warp][mid] <= u) lo = mid; else hi = mid;
                    }
                    const SegRecB& q = s_seg[warp][lo];
                    int k = u - s_pre[warp][lo];
                    real dt = (q.t1 - q.t0) / (real)q.m;
                    real ta = q.t0 + dt * (real)k;
                    real tz = (k == q.m - 1) ? q.t1 : ta + dt;
                    const KGrid& G = B.grids[q.scene];
                    int nv = walk_range(G, G.tally + (size_t)q.slot * 2 * G.nvox, q.p, q.d, ta, tz, q.wk, q.wh);
                    c_vox += max(nv - (k > 0 ? 1 : 0), 0);   // a cut voxel is one visit
                }
                __syncwarp();
                if (c_vox >= COUNTER_FLUSH) {
                    atomicAdd(&s_cnt[1], (unsigned long long)c_vox);
                    c_vox = 0;
                }
            }
        }

        // ---- phase 3 ----
        bool ended = false, esc = false, absd = false;
        if (go) {
            const DevMaterial& M = T.mats[mat];
            p[0] += d[0] * s; p[1] += d[1] * s; p[2] += d[2] * s;
            if (!interact) {
                tau -= tau_b;
                if (escape) { esc = true; ended = true; }
                mat = -1;
            } else {
                phys ph, co, ra;
                parts(T, M, L, ph, co, ra);
                phys r = uni(rng) * (ph + co + ra);
                ++nsc;
                const int kind = r < ph ? 0 : (r < ph + co ? 1 : 2);
                // element draw, new direction and new free path outside the
                // branches: every interacting lane runs them together
                const int eslot = pick_element(T, M, L, kind, uni(rng));
                phys cost = P(1.0), e_new = E;
                bool ok = true;
                if (kind == 0) {
                    const phys e_line = sample_k_line(T.elems[eslot], E, fluorescence, rng);
                    if (e_line > P(0.0)) {
                        atomicAdd(B.scene_cnt + 4 * (size_t)sc + 3, 1ull);   // rare: K lines of heavy elements
                        e_new = e_line;
                    } else {
                        absd = true;
                        ended = true;
                    }
                } else if (kind == 1) {
                    phys eps;
                    sample_compton(T.sq + (size_t)eslot * TABLE_N, E, rng, eps, cost);
                    e_new = E * eps;
                } else if (!sample_rayleigh(T.rx + (size_t)eslot * TABLE_N, T.ra + (size_t)eslot * TABLE_N,
                                            T.ray_bucket + (size_t)eslot * (RAY_BUCKETS + 1),
                                            T.elems[eslot].ray_scale, E, rng, cost)) {
                    atomicOr(R.status, ST_RAYLEIGH_Q);
                    ended = true;
                    ok = false;
                }
                if (ok && !ended) {
                    if (kind == 0) isotropic(d, rng);                   // the fluorescence photon
                    else scatter_direction(d, cost, TWO_PI * uni(rng));
                    E = e_new;
                    tau = -p_log(uni(rng));
                }
                mat = -1;
            }
            if (!ended && steps >= R.max_steps) {
                atomicOr(R.status, ST_STEPS);
                ended = true;
            }
        }
        add_scene_counts(B, ended, sc, absd ? 1u : 0u, esc ? 1u : 0u, ended ? (unsigned)nsc : 0u, 0u, lane);
        if (ended) {
            c_steps += (unsigned)steps;
            live = false;
            if ((c_steps | c_vox) >= COUNTER_FLUSH) {
                atomicAdd(&s_cnt[0], (unsigned long long)c_steps);
                atomicAdd(&s_cnt[1], (unsigned long long)c_vox);
                c_steps = c_vox = 0;
            }
        }
    }
    atomicAdd(&s_cnt[0], (unsigned long long)c_steps);
    atomicAdd(&s_cnt[1], (unsigned long long)c_vox);
    __syncthreads();
    if (threadIdx.x < 2) atomicAdd(R.counters + 4 + threadIdx.x, s_cnt[threadIdx.x]);
}

// Batch statistics fold (tally.py:59-94): T += S, Q += S^2/n_b,
// n_hit += (S_k != 0 or S_h != 0), S = 0.
// (A scratch cell is read as FP32 pairs when cell32; the cell is zeroed
// whole either way.)
__device__ __forceinline__ double2 cell_read(const double2* scratch, long long i, int cell32) {
    if (cell32) {
        const float2 f = reinterpret_cast<const float2*>(scratch)[2 * i];
        return make_double2((double)f.x, (double)f.y);
    }
    return scratch[i];
}

__global__ void fold_kernel(double2* __restrict__ total, double2* __restrict__ q,
                            int* __restrict__ nhit, double2* __restrict__ scratch,
                            long long nvox, double inv_nb, int cell32) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < nvox; i += stride) {
        double2 s = cell_read(scratch, i, cell32);
        if (s.x != 0.0 || s.y != 0.0) {
            double2 t = total[i];
            t.x += s.x; t.y += s.y;
            total[i] = t;
            double2 qq = q[i];
            qq.x += s.x * s.x * inv_nb;
            qq.y += s.y * s.y * inv_nb;
            q[i] = qq;
            nhit[i] += 1;
            scratch[i] = make_double2(0.0, 0.0);
        }
    }
}

// The batches of one launch at once (slots 0..n-1 in order, each as
// fold_kernel): the totals, sums of squares and hit counts of a voxel are
// read and written once per launch instead of once per batch.  The
// additions per voxel happen in the same order as slot-by-slot folds.
struct FoldSlots {
    double inv_nb[MAX_SCRATCH];     // 1 / histories of each batch; 0 skips the slot
    int n;
};

__global__ void fold_slots_kernel(double2* __restrict__ total, double2* __restrict__ q, int* __restrict__ nhit,
                                  double2* __restrict__ scratch, long long nvox, const FoldSlots F, int cell32) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < nvox; i += stride) {
        double2 t = make_double2(0.0, 0.0), qq = make_double2(0.0, 0.0);
        int h = 0;
        bool loaded = false;
        for (int s = 0; s < F.n; ++s) {
            if (F.inv_nb[s] == 0.0) continue;
            double2* sc = scratch + (size_t)s * nvox;
            const double2 v = cell_read(sc, i, cell32);
            if (v.x != 0.0 || v.y != 0.0) {
                if (!loaded) { t = total[i]; qq = q[i]; h = nhit[i]; loaded = true; }
                t.x += v.x; t.y += v.y;
                qq.x += v.x * v.x * F.inv_nb[s];
                qq.y += v.y * v.y * F.inv_nb[s];
                h += 1;
                sc[i] = make_double2(0.0, 0.0);
            }
        }
        if (loaded) { total[i] = t; q[i] = qq; nhit[i] = h; }
    }
}

// Slots 0..n-1 into the totals without statistics, in order: T += S_s, S_s = 0.
__global__ void fold_plain_slots_kernel(double2* __restrict__ total, double2* __restrict__ scratch, long long nvox,
                                        int n_slots, int cell32) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < nvox; i += stride) {
        double2 t = make_double2(0.0, 0.0);
        bool loaded = false;
        for (int s = 0; s < n_slots; ++s) {
            double2* sc = scratch + (size_t)s * nvox;
            const double2 v = cell_read(sc, i, cell32);
            if (v.x != 0.0 || v.y != 0.0) {
                if (!loaded) { t = total[i]; loaded = true; }
                t.x += v.x;
                t.y += v.y;
                sc[i] = make_double2(0.0, 0.0);
            }
        }
        if (loaded) total[i] = t;
    }
}

// Batch scratch into the totals without statistics: T += S, S = 0.
__global__ void fold_plain_kernel(double2* __restrict__ total, double2* __restrict__ scratch, long long nvox,
                                  int cell32) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < nvox; i += stride) {
        double2 s = cell_read(scratch, i, cell32);
        if (s.x != 0.0 || s.y != 0.0) {
            double2 t = total[i];
            t.x += s.x;
            t.y += s.y;
            total[i] = t;
            scratch[i] = make_double2(0.0, 0.0);
        }
    }
}

// Split the interleaved device grids into the caller's separate arrays
// (totals include a pending, not yet folded batch, as VoxelGrid.kerma_keV does).
__global__ void unpack_kernel(const double2* __restrict__ total, const double2* __restrict__ pending,
                              const double2* __restrict__ q, const int* __restrict__ nhit,
                              double* __restrict__ ok, double* __restrict__ oh, double* __restrict__ ok2,
                              double* __restrict__ oh2, int* __restrict__ on, long long nvox) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < nvox; i += stride) {
        double2 x = total[i];
        if (pending) { double2 y = pending[i]; x.x += y.x; x.y += y.y; }
        ok[i] = x.x;
        oh[i] = x.y;
        if (q) { double2 z = q[i]; ok2[i] = z.x; oh2[i] = z.y; on[i] = nhit[i]; }
    }
}

// ---------------------------------------------------------------------------
// output maps (chatcarlo/diagnostics.py:16-26, tally.py:109-132, 135-175)
// ---------------------------------------------------------------------------

// One primitive in FP64 for the point test at voxel centres
// (geometry.py:102-118 closed containment; an ellipsoid as (p-c)/semi).
struct MapPrim {
    int type, axis;
    double c[3], s[3];      // centre; box / ellipsoid full edge or axis lengths
    double r, height;       // sphere, cylinder
    double density;         // of the primitive's material, g/cm^3
};

struct KMaps {
    double o[3], h;         // grid origin and voxel edge (cm)
    int nx, ny, nz;
    double volume;          // voxel volume, computed by the caller as h ** 3
    double divisor;         // every map is divided by it last (1, or the history count)
    double bg_density;
    double n_hist, n_batches_minus_1;
    int rel_defined;        // M >= 2 and N > 0
    int n_prims;
};

// Products and sums rounded one by one (no contraction into FMAs), in the
// order NumPy evaluates the same expressions, so the maps equal the host's.
__device__ __forceinline__ double sq_rn(double x) { return __dmul_rn(x, x); }

__device__ __forceinline__ bool map_contains(const MapPrim& g, const double p[3]) {
    if (g.type == CC_SHAPE_BOX) {
        bool in = true;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double half = __dmul_rn(g.s[k], 0.5);          // s / 2 (exact)
            in = in && p[k] >= __dsub_rn(g.c[k], half) && p[k] <= __dadd_rn(g.c[k], half);
        }
        return in;
    }
    if (g.type == CC_SHAPE_SPHERE) {
        double d2 = __dadd_rn(__dadd_rn(sq_rn(__dsub_rn(p[0], g.c[0])), sq_rn(__dsub_rn(p[1], g.c[1]))),
                              sq_rn(__dsub_rn(p[2], g.c[2])));
        return d2 <= sq_rn(g.r);
    }
    if (g.type == CC_SHAPE_ELLIPSOID) {
        double u[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) u[k] = __ddiv_rn(__dsub_rn(p[k], g.c[k]), __dmul_rn(g.s[k], 0.5));
        return __dadd_rn(__dadd_rn(sq_rn(u[0]), sq_rn(u[1])), sq_rn(u[2])) <= 1.0;
    }
    const int a = g.axis;
    const int o0 = a == 0 ? 1 : 0, o1 = a == 2 ? 1 : 2;
    const double r2 = __dadd_rn(sq_rn(__dsub_rn(comp(p, o0), comp(g.c, o0))), sq_rn(__dsub_rn(comp(p, o1), comp(g.c, o1))));
    return r2 <= sq_rn(g.r) && fabs(__dsub_rn(comp(p, a), comp(g.c, a))) <= __dmul_rn(g.height, 0.5);
}

__global__ void maps_kernel(const double2* __restrict__ total, const double2* __restrict__ pending,
                            const double2* __restrict__ q, const MapPrim* __restrict__ prims, const KMaps M,
                            double* __restrict__ dose, double* __restrict__ h10, double* __restrict__ krel,
                            double* __restrict__ hrel) {
    const long long nvox = (long long)M.nx * M.ny * M.nz;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
         v += (long long)gridDim.x * blockDim.x) {
        double2 t = total[v];
        if (pending) { const double2 y = pending[v]; t.x += y.x; t.y += y.y; }
        if (dose) {
            const int iz = (int)(v % M.nz), iy = (int)((v / M.nz) % M.ny), ix = (int)(v / ((long long)M.ny * M.nz));
            const double p[3] = {__dadd_rn(M.o[0], __dmul_rn((double)ix + 0.5, M.h)),
                                 __dadd_rn(M.o[1], __dmul_rn((double)iy + 0.5, M.h)),
                                 __dadd_rn(M.o[2], __dmul_rn((double)iz + 0.5, M.h))};
            double rho = M.bg_density;                         // the last primitive holding the centre wins
            for (int i = 0; i < M.n_prims; ++i)
                if (map_contains(prims[i], p)) rho = prims[i].density;
            const double mass = __dmul_rn(__dmul_rn(rho, M.volume), 1e-3);
            const double energy = __dmul_rn(__dmul_rn(t.x, 1e-3), 1.602176634e-13);
            dose[v] = __ddiv_rn(mass > 0.0 ? __ddiv_rn(energy, mass) : 0.0, M.divisor);
        }
        if (h10) h10[v] = __ddiv_rn(__ddiv_rn(t.y, M.volume), M.divisor);
        if (krel || hrel) {
            const double2 s2 = q[v];
            const double T[2] = {t.x, t.y}, Q[2] = {s2.x, s2.y};
            double r[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                if (!M.rel_defined) { r[j] = CUDART_NAN; continue; }
                double var = __ddiv_rn(__dsub_rn(Q[j], __ddiv_rn(sq_rn(T[j]), M.n_hist)), M.n_batches_minus_1);
                var = var < 0.0 ? 0.0 : var;                      // np.clip(var, 0, None); NaN stays NaN
                const double sem = __dsqrt_rn(__ddiv_rn(var, M.n_hist));
                const double mean = __ddiv_rn(T[j], M.n_hist);
                r[j] = mean != 0.0 ? __ddiv_rn(sem, mean) : CUDART_NAN;
            }
            if (krel) krel[v] = r[0];
            if (hrel) hrel[v] = r[1];
        }
    }
}

__global__ void sample_source_kernel(const KSource SRC, long long n, long long first,
                                     unsigned long long seed, double* pos, double* dir, double* en) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    HistoryRng rng;
    rng.init(seed, (unsigned long long)(first + i), 0u);
    real p[3], d[3];
    phys E;
    sample_source<true>(SRC, rng, p, d, E);
    for (int k = 0; k < 3; ++k) { pos[3 * i + k] = p[k]; dir[3 * i + k] = d[k]; }
    en[i] = E;
}

// One interaction per thread through the transport kernel's own device
// functions: the element draw of the interaction kind, then the photoelectric
// K-line draw, the bound-Compton sampler or the Rayleigh sampler.  Photon i
// draws the Philox stream of history i under the seed.
constexpr int INTERACT_PHOTO = 0, INTERACT_COMPTON = 1, INTERACT_RAYLEIGH = 2;

__global__ void interaction_kernel(const KTables T, int kind, long long n, const int* __restrict__ mat,
                                   const phys* __restrict__ energy, unsigned long long seed, int fluorescence,
                                   double* out_a, double* out_b, int* out_z, unsigned* status) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = mat[i];
    const phys E = energy[i];
    out_a[i] = 0.0;
    out_b[i] = 0.0;
    out_z[i] = 0;
    if (m < 0 || m >= T.n_mat) { atomicOr(status, ST_BOUNDS); return; }
    if (!(E >= E_MIN_KEV && E <= E_MAX_KEV)) { atomicOr(status, ST_ENERGY); return; }
    HistoryRng rng;
    rng.init(seed, (unsigned long long)i, 0u);
    const DevMaterial& M = T.mats[m];
    const Lookup L = energy_index(T, M, p_log(E));
    const int slot = pick_element(T, M, L, kind, uni(rng));
    out_z[i] = T.elems[slot].z;
    if (kind == INTERACT_PHOTO) {
        out_a[i] = sample_k_line(T.elems[slot], E, fluorescence, rng);
    } else if (kind == INTERACT_COMPTON) {
        phys eps, cost;
        sample_compton(T.sq + (size_t)slot * TABLE_N, E, rng, eps, cost);
        out_a[i] = eps;
        out_b[i] = cost;
    } else {
        phys cost;
        if (!sample_rayleigh(T.rx + (size_t)slot * TABLE_N, T.ra + (size_t)slot * TABLE_N,
                             T.ray_bucket + (size_t)slot * (RAY_BUCKETS + 1), T.elems[slot].ray_scale, E, rng,
                             cost)) {
            atomicOr(status, ST_RAYLEIGH_Q);
            return;
        }
        out_a[i] = cost;
    }
}

// Raw Philox4x32-10 blocks (known-answer tests of the generator).
__global__ void philox_kernel(long long n, const uint32_t* __restrict__ ctr, const uint32_t* __restrict__ key,
                              uint32_t* __restrict__ out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32x4 r = philox_block(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3], key[2 * i],
                                 key[2 * i + 1]);
    out[4 * i] = r.x;
    out[4 * i + 1] = r.y;
    out[4 * i + 2] = r.z;
    out[4 * i + 3] = r.w;
}

}  // namespace cc

// ===========================================================================
// host side: objects and the C ABI
// ===========================================================================

using namespace cc;

static thread_local std::string g_last_error;

static int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CC_CUDA(call)                                                                 \
    do {                                                                              \
        cudaError_t _e = (call);                                                      \
        if (_e != cudaSuccess)                                                        \
            return set_error(CC_E_DEVICE, std::string(#call ": ") + cudaGetErrorString(_e)); \
    } while (0)

struct cc_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t kev0 = nullptr, kev1 = nullptr;     // around the transport kernel alone
    double* d_edep = nullptr;                       // [MAX_SCRATCH * MAX_MATS] per-launch reductions
    char* d_io = nullptr;                           // staging of cc_transport_photons (grow-only)
    size_t io_bytes = 0;
    unsigned* d_status = nullptr;
    unsigned long long* d_counters = nullptr;   // [5] + work counter
    int block = 256;
    int blocks_per_sm = 0;                       // 0 = occupancy based
    int tally_blocks_per_sm = 1;                 // resident tally_kernel blocks per SM
    long long max_steps = 100000;
    int tally_fp32 = 0;                          // 1: FP32 scratch cells for slots of <= FP32_SLOT_HISTORIES
    // cc_run keeps up to LAUNCH_RING launches in flight; each one's
    // reductions land in its own page-locked record
    static constexpr int LAUNCH_RING = 3;
    struct LaunchRec {
        double* h_edep = nullptr;                // [MAX_SCRATCH * MAX_MATS]
        unsigned long long* h_cnt = nullptr;     // [8] the launch's counters
        unsigned* h_status = nullptr;
        cudaEvent_t k0 = nullptr, k1 = nullptr;  // around the transport kernel
        cudaEvent_t done = nullptr;              // after the copies into this record
        int ns = 0;                              // batches of the launch
        long long n = 0;                         // histories of the launch
        long long seg_cap = 0;                   // its segment-queue capacity
        bool busy = false;
    } ring[LAUNCH_RING];
    char* h_ring = nullptr;
    // deferred tally's segment queue (grow-only) and the records per history
    // to provide for, raised when a launch offers more than its capacity
    SegRec* d_seg = nullptr;
    long long seg_alloc = 0;
    double seg_per_history = 8.0;
    int tally_queue = 0;                         // cc_ctx_set_tally_queue
    long long tally_queue_cap = 0;               // fixed capacity (records), 0 = automatic
    // copy streams and events of cc_transport_photons' chunked pipeline
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t ev_in[LAUNCH_RING] = {}, ev_k[LAUNCH_RING] = {};
};

struct cc_tables {
    cc_ctx* ctx;
    KTables k;
    std::vector<void*> allocs;
    int n_mat;
};

struct cc_scene {
    cc_ctx* ctx;
    KScene k;
};

struct cc_source {
    cc_ctx* ctx;
    KSource k;
    std::vector<void*> allocs;
};

struct cc_grid {
    cc_ctx* ctx;
    KGrid k;
    int flags;
    double* d_total = nullptr;      // double2 per voxel
    double* d_q = nullptr;
    int* d_nhit = nullptr;
    double* d_scratch = nullptr;    // [n_scratch][nvox] double2; slot 0 is the pending batch
    int n_scratch = 0;
    char* d_out = nullptr;          // download staging: kerma, h10, kerma_sum2, h10_sum2 (f64), n_hit (i32)
    double* d_maps = nullptr;       // cc_grid_maps staging: 4 maps (f64), allocated on first use
    double origin64[3] = {0, 0, 0}; // the caller's FP64 origin and voxel edge (the kernels track in FP32)
    double voxel64 = 0;
    char* h_out = nullptr;          // pinned host copy of d_out
    long long n_batches = 0;
    long long n_histories = 0;
};

template <class T>
static int dev_upload(std::vector<void*>& allocs, const std::vector<T>& v, const T** out) {
    void* p = nullptr;
    size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
    CC_CUDA(cudaMalloc(&p, bytes));
    allocs.push_back(p);
    if (!v.empty()) CC_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    *out = (const T*)p;
    return CC_OK;
}

template <bool FS, bool TL, bool HEEL = false>
static cudaError_t launch_transport(cc_ctx* c, const KTables& T, const KScene& S, const KGrid& G,
                                    const KSource& SRC, const KRun& R, size_t smem, int grid_blocks) {
    if constexpr (TL) {
        if (R.defer)
            transport_kernel<FS, TL, HEEL, TV_DEFER><<<grid_blocks, c->block, smem, c->stream>>>(T, S, G, SRC, R);
        else if (G.tally32)
            transport_kernel<FS, TL, HEEL, CELL_FP32><<<grid_blocks, c->block, smem, c->stream>>>(T, S, G, SRC, R);
        else
            transport_kernel<FS, TL, HEEL, CELL_FP64><<<grid_blocks, c->block, smem, c->stream>>>(T, S, G, SRC, R);
    } else {
        transport_kernel<FS, TL, HEEL><<<grid_blocks, c->block, smem, c->stream>>>(T, S, G, SRC, R);
    }
    return cudaGetLastError();
}

extern "C" {

int cc_version(void) { return CC_ABI_VERSION; }

const char* cc_last_error(void) { return g_last_error.c_str(); }

int cc_ctx_create(int device, cc_ctx** out) {
    if (!out) return set_error(CC_E_INVALID, "out is NULL");
    cc_ctx* c = new (std::nothrow) cc_ctx();
    if (!c) return set_error(CC_E_NOMEM, "out of host memory");
    c->device = device;
    CC_CUDA(cudaSetDevice(device));
    CC_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    CC_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CC_CUDA(cudaEventCreate(&c->ev0));
    CC_CUDA(cudaEventCreate(&c->ev1));
    CC_CUDA(cudaEventCreate(&c->kev0));
    CC_CUDA(cudaEventCreate(&c->kev1));
    {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, tally_kernel, BLOCK, 0) == cudaSuccess && occ > 0)
            c->tally_blocks_per_sm = occ;
    }
    CC_CUDA(cudaMalloc(&c->d_edep, (size_t)MAX_SCRATCH * MAX_MATS * sizeof(double)));
    CC_CUDA(cudaMalloc(&c->d_status, sizeof(unsigned)));
    CC_CUDA(cudaMalloc(&c->d_counters, 8 * sizeof(unsigned long long)));
    *out = c;
    return CC_OK;
}

int cc_ctx_destroy(cc_ctx* c) {
    if (!c) return CC_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    cudaFree(c->d_status);
    cudaFree(c->d_counters);
    cudaFree(c->d_edep);
    cudaFree(c->d_io);
    for (auto& r : c->ring) {
        if (r.k0) cudaEventDestroy(r.k0);
        if (r.k1) cudaEventDestroy(r.k1);
        if (r.done) cudaEventDestroy(r.done);
    }
    cudaFreeHost(c->h_ring);
    cudaFree(c->d_seg);
    for (int i = 0; i < cc_ctx::LAUNCH_RING; ++i) {
        if (c->ev_in[i]) cudaEventDestroy(c->ev_in[i]);
        if (c->ev_k[i]) cudaEventDestroy(c->ev_k[i]);
    }
    if (c->s_in) cudaStreamDestroy(c->s_in);
    if (c->s_out) cudaStreamDestroy(c->s_out);
    cudaEventDestroy(c->ev0);
    cudaEventDestroy(c->ev1);
    cudaEventDestroy(c->kev0);
    cudaEventDestroy(c->kev1);
    cudaStreamDestroy(c->stream);
    delete c;
    return CC_OK;
}

int cc_ctx_set_launch(cc_ctx* c, int block_size, int blocks_per_sm) {
    if (!c) return set_error(CC_E_INVALID, "ctx is NULL");
    if (block_size != 0 && (block_size % 32 != 0 || block_size > 256 || block_size < 32))
        return set_error(CC_E_INVALID, "block_size must be a multiple of 32 in [32, 256]");
    if (blocks_per_sm < 0 || blocks_per_sm > 64) return set_error(CC_E_INVALID, "blocks_per_sm out of range");
    c->block = block_size ? block_size : 256;
    c->blocks_per_sm = blocks_per_sm;
    return CC_OK;
}

int cc_ctx_set_step_limit(cc_ctx* c, int64_t max_steps) {
    if (!c || max_steps <= 0 || max_steps > (1LL << 30))
        return set_error(CC_E_INVALID, "step limit must be in [1, 2^30]");
    c->max_steps = max_steps;
    return CC_OK;
}

int cc_ctx_set_tally_queue(cc_ctx* c, int32_t on, int64_t capacity) {
    if (!c || capacity < 0) return set_error(CC_E_INVALID, "NULL context or negative capacity");
    c->tally_queue = on ? 1 : 0;
    c->tally_queue_cap = capacity;
    return CC_OK;
}

int cc_ctx_set_tally_fp32(cc_ctx* c, int32_t on) {
    if (!c) return set_error(CC_E_INVALID, "NULL context");
    c->tally_fp32 = on ? 1 : 0;
    return CC_OK;
}

// ---------------------------------------------------------------------------

int cc_tables_create(cc_ctx* ctx, const cc_table_desc* desc, cc_tables** out) {
    if (!ctx || !desc || !out) return set_error(CC_E_INVALID, "NULL argument");
    if (desc->n_materials < 1 || desc->n_materials > MAX_MATS)
        return set_error(CC_E_INVALID, "n_materials must be in [1, 16]");
    if (desc->n_elements < 1 || desc->n_elements > MAX_ELEMS)
        return set_error(CC_E_INVALID, "n_elements must be in [1, 48]");
    CC_CUDA(cudaSetDevice(ctx->device));
    std::vector<phys> loge, elem_cum;
    std::vector<PNode> nodes;
    std::vector<unsigned short> bucket;
    std::vector<DevMaterial> mats(desc->n_materials);
    for (int m = 0; m < desc->n_materials; ++m) {
        const cc_material_desc& md_ = desc->materials[m];
        if (md_.n_nodes < 2 || md_.n_nodes > 65535 || md_.n_elements < 1 || md_.n_elements > MAX_ELEMS_PER_MAT ||
            !md_.log_tally)
            return set_error(CC_E_INVALID, "material " + std::to_string(m) + ": bad sizes");
        DevMaterial& dm = mats[m];
        memset(&dm, 0, sizeof(dm));
        dm.density = (phys)md_.density;
        dm.n_nodes = md_.n_nodes;
        dm.n_el = md_.n_elements;
        dm.node_off = (int)loge.size();
        dm.elem_off = (int)elem_cum.size();
        dm.bucket_off = (int)bucket.size();
        double lmax = log(150.0);
        dm.bucket_scale = (phys)(N_BUCKETS / lmax);
        for (int i = 0; i < md_.n_nodes; ++i) {
            if (i > 0 && !(md_.log_e[i] > md_.log_e[i - 1]))
                return set_error(CC_E_INVALID, "material " + std::to_string(m) + ": log_e not increasing");
            loge.push_back((phys)md_.log_e[i]);
            const double* q = md_.log_parts + 4 * (size_t)i;
            const double* t = md_.log_tally + 2 * (size_t)i;
            nodes.push_back(PNode{(phys)md_.log_e[i], (phys)q[0], (phys)q[1], (phys)q[2]});
            nodes.push_back(PNode{(phys)q[3], (phys)t[0], (phys)t[1], (phys)0});
        }
        // node index per bucket: last node whose (table-precision) log E <= the bucket start
        int node = 0;
        const phys* lf = loge.data() + dm.node_off;
        for (int b = 0; b < N_BUCKETS; ++b) {
            phys start = (phys)b / dm.bucket_scale;
            while (node + 1 < md_.n_nodes - 1 && lf[node + 1] <= start) ++node;
            bucket.push_back((unsigned short)node);
        }
        {
            // per kind k and node: normalised cumulative sums of w_i sigma_i (FP64)
            const int ne = md_.n_elements, nn = md_.n_nodes;
            std::vector<double> w(ne);
            for (int k = 0; k < 3; ++k) {
                size_t base = elem_cum.size();
                elem_cum.resize(base + (size_t)(ne - 1) * nn);
                for (int j = 0; j < nn; ++j) {
                    double tot = 0.0;
                    for (int e = 0; e < ne; ++e) {
                        w[e] = exp(md_.log_elem[((size_t)e * 3 + k) * nn + j]);
                        tot += w[e];
                    }
                    double acc = 0.0;
                    for (int e = 0; e < ne - 1; ++e) {
                        acc += w[e];
                        elem_cum[base + (size_t)e * nn + j] = (phys)(tot > 0.0 ? acc / tot : 1.0);
                    }
                }
            }
        }
        for (int e = 0; e < md_.n_elements; ++e) {
            int slot = md_.element_slot[e];
            if (slot < 0 || slot >= desc->n_elements)
                return set_error(CC_E_INVALID, "material element slot out of range");
            dm.el_slot[e] = slot;
        }
    }
    std::vector<DevElement> els(desc->n_elements);
    std::vector<phys> sq, rx, ra;
    std::vector<int> rbk;
    for (int e = 0; e < desc->n_elements; ++e) {
        const cc_element_desc& ed = desc->elements[e];
        if (ed.n_lines < 0 || ed.n_lines > 8) return set_error(CC_E_INVALID, "n_lines must be <= 8");
        DevElement& de = els[e];
        memset(&de, 0, sizeof(de));
        de.k_edge = (phys)ed.k_edge_kev;
        de.k_prob = (phys)ed.k_shell_prob;
        de.omega = (phys)ed.omega_k;
        de.n_lines = ed.n_lines;
        de.emits = ed.emits && ed.n_lines > 0;
        de.z = ed.z;
        double cum = 0.0;
        for (int k = 0; k < ed.n_lines; ++k) {
            cum += ed.line_p[k];
            de.line_e[k] = (phys)ed.line_e[k];
            de.line_cum[k] = (phys)cum;
        }
        size_t ra_off = ra.size();
        for (int i = 0; i < TABLE_N; ++i) {
            if (i > 0 && !(ed.ray_a[i] >= ed.ray_a[i - 1]))
                return set_error(CC_E_INVALID, "Rayleigh A(x) table must not decrease");
            sq.push_back((phys)ed.s_over_z[i]);
            rx.push_back((phys)ed.ray_x[i]);
            ra.push_back((phys)ed.ray_a[i]);
        }
        // bucket index on the FP32 table the kernel searches
        const phys a_end = ra[ra_off + TABLE_N - 1];
        if (!(a_end > 0.0f)) return set_error(CC_E_INVALID, "Rayleigh A(x) table is empty");
        de.ray_scale = (phys)RAY_BUCKETS / a_end;
        int row = 0;
        for (int b = 0; b <= RAY_BUCKETS; ++b) {
            phys start = (phys)b / de.ray_scale;
            while (row + 1 < TABLE_N - 1 && ra[ra_off + row + 1] <= start) ++row;
            rbk.push_back(row);
        }
    }

    cc_tables* t = new (std::nothrow) cc_tables();
    if (!t) return set_error(CC_E_NOMEM, "out of host memory");
    t->ctx = ctx;
    t->n_mat = desc->n_materials;
    KTables& k = t->k;
    int rc;
#define UP(vec, field) if ((rc = dev_upload(t->allocs, vec, &k.field)) != CC_OK) { cc_tables_destroy(t); return rc; }
    UP(nodes, nodes);
    UP(elem_cum, elem_cum);
    UP(bucket, bucket);
    UP(mats, mats);
    UP(els, elems);
    UP(sq, sq);
    UP(rx, rx);
    UP(ra, ra);
    UP(rbk, ray_bucket);
#undef UP
    k.n_mat = desc->n_materials;
    k.n_elem = desc->n_elements;
    *out = t;
    return CC_OK;
}

int cc_tables_destroy(cc_tables* t) {
    if (!t) return CC_OK;
    cudaSetDevice(t->ctx->device);
    for (void* p : t->allocs) cudaFree(p);
    delete t;
    return CC_OK;
}

int cc_scene_create(cc_ctx* ctx, const cc_primitive* prims, int32_t n_prims, int32_t background,
                    const double world_lo[3], const double world_hi[3], cc_scene** out) {
    if (!ctx || !out || !world_lo || !world_hi || (n_prims > 0 && !prims))
        return set_error(CC_E_INVALID, "NULL argument");
    if (n_prims < 0 || n_prims > MAX_PRIMS) return set_error(CC_E_INVALID, "n_prims must be in [0, 64]");
    if (background < 0 || background >= MAX_MATS) return set_error(CC_E_UNKNOWN_MATERIAL, "background material out of range");
    cc_scene* s = new (std::nothrow) cc_scene();
    if (!s) return set_error(CC_E_NOMEM, "out of host memory");
    s->ctx = ctx;
    KScene& k = s->k;
    memset(&k, 0, sizeof(k));
    k.n_prims = n_prims;
    k.background = background;
    double extent = 1.0;
    for (int a = 0; a < 3; ++a) {
        k.wlo[a] = (real)world_lo[a];
        k.whi[a] = (real)world_hi[a];
        extent = std::max(extent, std::max(fabs(world_lo[a]), fabs(world_hi[a])));
    }
    // 8 ulps of the largest world coordinate, and at least the 1e-6 cm of
    // transport.py:155 / geometry.py:214
#ifdef CC_TRACK_FP64
    k.eps = (real)1e-6;
#else
    k.eps = (float)std::max(1e-6, 8.0 * extent * 5.960464477539063e-08);
#endif
    for (int i = 0; i < n_prims; ++i) {
        const cc_primitive& p = prims[i];
        DevPrim& g = k.prims[i];
        if (p.type < 0 || p.type > 3) { delete s; return set_error(CC_E_BAD_SHAPE, "unknown primitive type " + std::to_string(p.type)); }
        if (p.type == CC_SHAPE_ELLIPSOID && !(p.size[0] > 0 && p.size[1] > 0 && p.size[2] > 0)) {
            delete s;
            return set_error(CC_E_INVALID, "ellipsoid axes must be positive");
        }
        if (p.material < 0 || p.material >= MAX_MATS) { delete s; return set_error(CC_E_UNKNOWN_MATERIAL, "primitive material out of range"); }
        if (p.type == CC_SHAPE_CYLINDER && (p.axis < 0 || p.axis > 2)) { delete s; return set_error(CC_E_INVALID, "cylinder axis must be 0, 1 or 2"); }
        g.type = p.type;
        g.material = p.material;
        g.axis = p.axis;
        for (int a = 0; a < 3; ++a) { g.c[a] = (real)p.center[a]; g.h[a] = (real)(0.5 * p.size[a]); }
        g.r2 = (real)(p.radius * p.radius);
        g.r = (real)p.radius;
        g.hh = (real)(0.5 * p.height);
        if (p.type == CC_SHAPE_ELLIPSOID)
            g.r = (real)(2.0 / std::min(p.size[0], std::min(p.size[1], p.size[2])));
    }
    *out = s;
    return CC_OK;
}

int cc_scene_destroy(cc_scene* s) {
    delete s;
    return CC_OK;
}

// Walker alias table of a discrete spectrum, built in FP64 and appended to
// (q, alias, energies); alias entries are indices into the appended tables.
// Returns CC_OK or the error of a bad spectrum.
static int append_alias_table(const double* e, const double* w, int n, std::vector<phys>& qf,
                              std::vector<int>& alias_out, std::vector<phys>& ef) {
    double tot = 0.0;
    for (int i = 0; i < n; ++i) {
        if (!(w[i] >= 0.0)) return set_error(CC_E_INVALID, "negative spectrum weight");
        if (!(e[i] >= 1.0 && e[i] <= 150.0))
            return set_error(CC_E_ENERGY_RANGE, "spectrum energy outside [1, 150] keV");
        tot += w[i];
    }
    if (!(tot > 0.0)) return set_error(CC_E_INVALID, "spectrum weights sum to zero");
    const int base = (int)ef.size();
    std::vector<double> q(n);
    std::vector<int> alias(n);
    std::vector<int> small, large;
    for (int i = 0; i < n; ++i) {
        q[i] = w[i] / tot * n;
        alias[i] = i;
        (q[i] < 1.0 ? small : large).push_back(i);
    }
    while (!small.empty() && !large.empty()) {
        int s = small.back(); small.pop_back();
        int l = large.back();
        alias[s] = l;
        q[l] = q[l] + q[s] - 1.0;
        if (q[l] < 1.0) { large.pop_back(); small.push_back(l); }
    }
    for (int i : large) q[i] = 1.0;
    for (int i : small) q[i] = 1.0;
    for (int i = 0; i < n; ++i) {
        qf.push_back((phys)q[i]);
        alias_out.push_back(base + alias[i]);
        ef.push_back((phys)e[i]);
    }
    return CC_OK;
}

int cc_source_create(cc_ctx* ctx, const cc_source_desc* d, cc_source** out) {
    if (!ctx || !d || !out) return set_error(CC_E_INVALID, "NULL argument");
    if (d->n_energies < 1 || !d->energies_kev || !d->weights) return set_error(CC_E_INVALID, "empty spectrum");
    if (d->field < 0 || d->field > 2) return set_error(CC_E_INVALID, "unknown field shape");
    CC_CUDA(cudaSetDevice(ctx->device));
    int n = d->n_energies;
    std::vector<phys> qf, ef;
    std::vector<int> alias;
    int rc0 = append_alias_table(d->energies_kev, d->weights, n, qf, alias, ef);
    if (rc0 != CC_OK) return rc0;
    // heel effect: per-bin alias tables behind one offset array
    const cc_heel_desc* hd = d->heel;
    std::vector<phys> hc, hf, hq, he;
    std::vector<int> ha, hoff;
    int heel_lo = 0, heel_hi = -1;
    if (hd) {
        if (d->field == CC_FIELD_PARALLEL) return set_error(CC_E_INVALID, "the heel effect needs a rect or cone field");
        if (hd->n_bins < 1 || hd->n_bins > CC_HEEL_MAX_BINS || !hd->centers || !hd->rel_fluence || !hd->bin_sizes ||
            !hd->energies_kev || !hd->weights || !(hd->span_cm > 0.0))
            return set_error(CC_E_INVALID, "heel: bad bins");
        int off = 0;
        for (int b = 0; b < hd->n_bins; ++b) {
            const double f = hd->rel_fluence[b];
            if (!(f >= 0.0 && f <= 1.0)) return set_error(CC_E_INVALID, "heel: relative fluence outside [0, 1]");
            if (b > 0 && !(hd->centers[b] > hd->centers[b - 1])) return set_error(CC_E_INVALID, "heel: centres not increasing");
            if (f > 0.0) { if (heel_hi < 0) heel_lo = b; heel_hi = b; }
            hc.push_back((phys)hd->centers[b]);
            hf.push_back((phys)f);
        }
        if (heel_hi < 0) return set_error(CC_E_INVALID, "heel: no bin has fluence");
        for (int b = 0; b < hd->n_bins; ++b) {
            const int nb = hd->bin_sizes[b];
            if (nb < 1) return set_error(CC_E_INVALID, "heel: empty bin spectrum");
            hoff.push_back((int)he.size());
            if (b >= heel_lo && b <= heel_hi) {
                // photons take energies only from the bins with fluence and those between
                int rc = append_alias_table(hd->energies_kev + off, hd->weights + off, nb, hq, ha, he);
                if (rc != CC_OK) return rc;
            } else {
                for (int i = 0; i < nb; ++i) { hq.push_back((phys)1); ha.push_back((int)he.size()); he.push_back((phys)1); }
            }
            off += nb;
        }
        hoff.push_back((int)he.size());
    }
    cc_source* s = new (std::nothrow) cc_source();
    if (!s) return set_error(CC_E_NOMEM, "out of host memory");
    s->ctx = ctx;
    KSource& k = s->k;
    k.field = d->field;
    k.rotation = d->rotation;
    k.rot_axis = d->rot_axis;
    k.n_angles = d->n_angles;
    for (int a = 0; a < 3; ++a) {
        k.pos[a] = (phys)d->position[a];
        k.dir[a] = (phys)d->direction[a];
        k.u[a] = (phys)d->u[a];
        k.v[a] = (phys)d->v[a];
        k.iso[a] = (phys)d->isocenter[a];
    }
    k.sid = (phys)d->sid_cm;
    k.su = (phys)d->size_u;
    k.sv = (phys)d->size_v;
    k.cos_half = (phys)d->cos_half_angle;
    k.scan = (phys)d->scan_length_cm;
    k.n_e = n;
    int rc;
    if ((rc = dev_upload(s->allocs, ef, &k.e)) != CC_OK) { cc_source_destroy(s); return rc; }
    if ((rc = dev_upload(s->allocs, qf, &k.alias_p)) != CC_OK) { cc_source_destroy(s); return rc; }
    if ((rc = dev_upload(s->allocs, alias, &k.alias_i)) != CC_OK) { cc_source_destroy(s); return rc; }
    k.heel_n = 0;
    if (hd) {
        k.heel_n = hd->n_bins;
        k.heel_lo = heel_lo;
        k.heel_hi = heel_hi;
        k.h_u = (phys)hd->h_u;
        k.h_v = (phys)hd->h_v;
        k.span = (phys)hd->span_cm;
        k.bin_w = (phys)(2.0 * hd->span_cm / hd->n_bins);
        if ((rc = dev_upload(s->allocs, hc, &k.heel_c)) != CC_OK ||
            (rc = dev_upload(s->allocs, hf, &k.heel_f)) != CC_OK ||
            (rc = dev_upload(s->allocs, hoff, &k.heel_off)) != CC_OK ||
            (rc = dev_upload(s->allocs, he, &k.heel_e)) != CC_OK ||
            (rc = dev_upload(s->allocs, hq, &k.heel_q)) != CC_OK ||
            (rc = dev_upload(s->allocs, ha, &k.heel_a)) != CC_OK) {
            cc_source_destroy(s);
            return rc;
        }
    }
    *out = s;
    return CC_OK;
}

int cc_source_destroy(cc_source* s) {
    if (!s) return CC_OK;
    cudaSetDevice(s->ctx->device);
    for (void* p : s->allocs) cudaFree(p);
    delete s;
    return CC_OK;
}

static int grid_alloc_scratch(cc_grid* g, int n) {
    if (g->n_scratch >= n) return CC_OK;
    double* p = nullptr;
    size_t bytes = (size_t)n * 2 * g->k.nvox * sizeof(double);
    CC_CUDA(cudaMalloc(&p, bytes));
    CC_CUDA(cudaMemsetAsync(p, 0, bytes, g->ctx->stream));
    if (g->d_scratch) {
        CC_CUDA(cudaMemcpyAsync(p, g->d_scratch, (size_t)g->n_scratch * 2 * g->k.nvox * sizeof(double),
                                cudaMemcpyDeviceToDevice, g->ctx->stream));
        CC_CUDA(cudaStreamSynchronize(g->ctx->stream));
        cudaFree(g->d_scratch);
    }
    g->d_scratch = p;
    g->n_scratch = n;
    return CC_OK;
}

int cc_grid_create(cc_ctx* ctx, const double origin[3], int32_t nx, int32_t ny, int32_t nz,
                   double voxel_cm, int32_t flags, cc_grid** out) {
    if (!ctx || !origin || !out) return set_error(CC_E_INVALID, "NULL argument");
    if (nx < 1 || ny < 1 || nz < 1 || !(voxel_cm > 0.0)) return set_error(CC_E_INVALID, "bad grid shape");
    if ((long long)nx * ny * nz >= (1LL << 31)) return set_error(CC_E_INVALID, "grids are limited to 2^31 - 1 voxels");
    CC_CUDA(cudaSetDevice(ctx->device));
    cc_grid* g = new (std::nothrow) cc_grid();
    if (!g) return set_error(CC_E_NOMEM, "out of host memory");
    g->ctx = ctx;
    g->flags = flags;
    KGrid& k = g->k;
    for (int a = 0; a < 3; ++a) { k.o[a] = (real)origin[a]; g->origin64[a] = origin[a]; }
    g->voxel64 = voxel_cm;
    k.h = (real)voxel_cm;
    k.inv_h = (real)(1.0 / voxel_cm);
    k.nx = nx; k.ny = ny; k.nz = nz;
    k.nvox = (long long)nx * ny * nz;
    k.enabled = 1;
    size_t b2 = (size_t)k.nvox * 2 * sizeof(double);
    if (cudaMalloc(&g->d_total, b2) != cudaSuccess) { delete g; return set_error(CC_E_NOMEM, "device allocation of the grid failed"); }
    if (flags & CC_GRID_STATS) {
        if (cudaMalloc(&g->d_q, b2) != cudaSuccess || cudaMalloc(&g->d_nhit, (size_t)k.nvox * sizeof(int)) != cudaSuccess) {
            cc_grid_destroy(g);
            return set_error(CC_E_NOMEM, "device allocation of the statistics grids failed");
        }
    }
    {
        int rc = grid_alloc_scratch(g, 1);           // every grid scores into batch scratch
        if (rc != CC_OK) { cc_grid_destroy(g); return rc; }
    }
    int rc = cc_grid_reset(g);
    if (rc != CC_OK) { cc_grid_destroy(g); return rc; }
    *out = g;
    return CC_OK;
}

int cc_grid_destroy(cc_grid* g) {
    if (!g) return CC_OK;
    cudaSetDevice(g->ctx->device);
    cudaFree(g->d_total);
    cudaFree(g->d_q);
    cudaFree(g->d_nhit);
    cudaFree(g->d_scratch);
    cudaFree(g->d_out);
    cudaFree(g->d_maps);
    cudaFreeHost(g->h_out);
    delete g;
    return CC_OK;
}

int cc_grid_reset(cc_grid* g) {
    if (!g) return set_error(CC_E_INVALID, "grid is NULL");
    cudaStream_t st = g->ctx->stream;
    size_t b2 = (size_t)g->k.nvox * 2 * sizeof(double);
    CC_CUDA(cudaMemsetAsync(g->d_total, 0, b2, st));
    if (g->d_q) CC_CUDA(cudaMemsetAsync(g->d_q, 0, b2, st));
    if (g->d_nhit) CC_CUDA(cudaMemsetAsync(g->d_nhit, 0, (size_t)g->k.nvox * sizeof(int), st));
    if (g->d_scratch) CC_CUDA(cudaMemsetAsync(g->d_scratch, 0, (size_t)g->n_scratch * b2, st));
    CC_CUDA(cudaStreamSynchronize(st));
    g->n_batches = 0;
    g->n_histories = 0;
    return CC_OK;
}

int cc_grid_device_buffers(cc_grid* g, double** totals, double** sum2s, int32_t** n_batches_hit,
                           int64_t* n_voxels, int64_t* n_batches, int64_t* n_histories) {
    if (!g) return set_error(CC_E_INVALID, "grid is NULL");
    // the grid's stream may still be writing the totals
    CC_CUDA(cudaSetDevice(g->ctx->device));
    CC_CUDA(cudaStreamSynchronize(g->ctx->stream));
    if (totals) *totals = g->d_total;
    if (sum2s) *sum2s = g->d_q;
    if (n_batches_hit) *n_batches_hit = (int32_t*)g->d_nhit;
    if (n_voxels) *n_voxels = g->k.nvox;
    if (n_batches) *n_batches = g->n_batches;
    if (n_histories) *n_histories = g->n_histories;
    return CC_OK;
}

int cc_grid_set_counts(cc_grid* g, int64_t n_batches, int64_t n_histories) {
    if (!g) return set_error(CC_E_INVALID, "grid is NULL");
    if (n_batches < 0 || n_histories < 0) return set_error(CC_E_INVALID, "negative count");
    g->n_batches = n_batches;
    g->n_histories = n_histories;
    return CC_OK;
}

// Histories a scratch slot may sum in FP32 cells (an opt-in of the context).
// Scores of unequal size round at random, ~sqrt(N) * 6e-8 relative after N
// of them; equal scores (a monoenergetic pencil beam's uncollided photons
// crossing the same voxels) round the same way each time, and at 2e5 such
// histories per slot the busiest voxels were seen 7e-4 apart between two
// summation orders.  Larger slots use FP64 cells; the FP64 build always does.
constexpr long long FP32_SLOT_HISTORIES = 1000000;

static int cell32_for(const cc_ctx* c, long long histories_per_slot) {
#ifdef CC_TRACK_FP64
    (void)c;
    (void)histories_per_slot;
    return 0;
#else
    return (c->tally_fp32 && histories_per_slot <= FP32_SLOT_HISTORIES) ? 1 : 0;
#endif
}

// Scratch slots [0, n_slots) into the totals without batch statistics.
static int fold_plain(cc_grid* g, int n_slots, int cell32) {
    cc_ctx* c = g->ctx;
    int threads = 256;
    int blocks = std::max(1, std::min((int)((g->k.nvox + threads - 1) / threads), c->sm_count * 8));
    if (n_slots > 1) {
        fold_plain_slots_kernel<<<blocks, threads, 0, c->stream>>>((double2*)g->d_total, (double2*)g->d_scratch,
                                                                   g->k.nvox, n_slots, cell32);
        CC_CUDA(cudaGetLastError());
        return CC_OK;
    }
    for (int s = 0; s < n_slots; ++s) {
        fold_plain_kernel<<<blocks, threads, 0, c->stream>>>(
            (double2*)g->d_total, (double2*)(g->d_scratch + (size_t)s * 2 * g->k.nvox), g->k.nvox, cell32);
        CC_CUDA(cudaGetLastError());
    }
    return CC_OK;
}

static int fold_batches(cc_grid* g, int n_slots, const long long* counts, int cell32) {
    cc_ctx* c = g->ctx;
    int threads = 256;
    int blocks = std::max(1, std::min((int)((g->k.nvox + threads - 1) / threads), c->sm_count * 8));
    if (n_slots > 1 && n_slots <= MAX_SCRATCH) {
        FoldSlots F;
        memset(&F, 0, sizeof(F));
        F.n = n_slots;
        for (int s = 0; s < n_slots; ++s) {
            if (counts[s] <= 0) continue;
            F.inv_nb[s] = 1.0 / (double)counts[s];
            g->n_batches += 1;
            g->n_histories += counts[s];
        }
        fold_slots_kernel<<<blocks, threads, 0, c->stream>>>((double2*)g->d_total, (double2*)g->d_q, g->d_nhit,
                                                             (double2*)g->d_scratch, g->k.nvox, F, cell32);
        CC_CUDA(cudaGetLastError());
        return CC_OK;
    }
    for (int s = 0; s < n_slots; ++s) {
        if (counts[s] <= 0) continue;
        fold_kernel<<<blocks, threads, 0, c->stream>>>(
            (double2*)g->d_total, (double2*)g->d_q, g->d_nhit,
            (double2*)(g->d_scratch + (size_t)s * 2 * g->k.nvox), g->k.nvox, 1.0 / (double)counts[s], cell32);
        CC_CUDA(cudaGetLastError());
        g->n_batches += 1;
        g->n_histories += counts[s];
    }
    return CC_OK;
}

int cc_grid_upload(cc_grid* g, const double* kerma, const double* h10, const double* k2, const double* h2,
                   const int32_t* nhit, int64_t n_batches, int64_t n_histories) {
    if (!g || !kerma || !h10) return set_error(CC_E_INVALID, "grid, kerma and h10 are required");
    const bool stats = g->d_q != nullptr;
    if (stats && (!k2 || !h2 || !nhit)) return set_error(CC_E_INVALID, "a statistics grid needs its sums of squares and hit counts");
    if (n_batches < 0 || n_histories < 0) return set_error(CC_E_INVALID, "negative batch or history count");
    cc_ctx* c = g->ctx;
    CC_CUDA(cudaSetDevice(c->device));
    const long long nv = g->k.nvox;
    std::vector<double> buf((size_t)2 * nv);
    for (long long i = 0; i < nv; ++i) { buf[2 * i] = kerma[i]; buf[2 * i + 1] = h10[i]; }
    CC_CUDA(cudaMemcpy(g->d_total, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (stats) {
        for (long long i = 0; i < nv; ++i) { buf[2 * i] = k2[i]; buf[2 * i + 1] = h2[i]; }
        CC_CUDA(cudaMemcpy(g->d_q, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice));
        CC_CUDA(cudaMemcpy(g->d_nhit, nhit, (size_t)nv * sizeof(int), cudaMemcpyHostToDevice));
    }
    if (g->d_scratch) CC_CUDA(cudaMemset(g->d_scratch, 0, (size_t)g->n_scratch * nv * 2 * sizeof(double)));
    g->n_batches = n_batches;
    g->n_histories = n_histories;
    return CC_OK;
}

int cc_grid_maps(cc_grid* g, const cc_primitive* prims, int32_t n_prims, const double* prim_density,
                 double background_density, double voxel_volume_cm3, double divisor, int32_t on_device,
                 double* dose_Gy, double* h10_pSv, double* kerma_rel, double* h10_rel) {
    if (!g) return set_error(CC_E_INVALID, "grid is NULL");
    if (n_prims < 0 || (n_prims > 0 && (!prims || !prim_density)))
        return set_error(CC_E_INVALID, "primitives and their densities are required");
    if (!(voxel_volume_cm3 > 0) || !(divisor > 0)) return set_error(CC_E_INVALID, "volume and divisor must be > 0");
    if ((kerma_rel || h10_rel) && !g->d_q) return set_error(CC_E_INVALID, "relative errors need a CC_GRID_STATS grid");
    cc_ctx* c = g->ctx;
    CC_CUDA(cudaSetDevice(c->device));
    std::vector<MapPrim> mp((size_t)n_prims);
    for (int i = 0; i < n_prims; ++i) {
        const cc_primitive& p = prims[i];
        if (p.type < 0 || p.type > 3) return set_error(CC_E_BAD_SHAPE, "unknown primitive type " + std::to_string(p.type));
        if (p.type == CC_SHAPE_CYLINDER && (p.axis < 0 || p.axis > 2)) return set_error(CC_E_INVALID, "cylinder axis must be 0, 1 or 2");
        MapPrim& m = mp[i];
        m.type = p.type;
        m.axis = p.axis;
        for (int a = 0; a < 3; ++a) { m.c[a] = p.center[a]; m.s[a] = p.size[a]; }
        m.r = p.radius;
        m.height = p.height;
        m.density = prim_density[i];
    }
    KMaps M;
    memset(&M, 0, sizeof(M));
    for (int a = 0; a < 3; ++a) M.o[a] = g->origin64[a];
    M.h = g->voxel64;
    M.nx = g->k.nx; M.ny = g->k.ny; M.nz = g->k.nz;
    M.volume = voxel_volume_cm3;
    M.divisor = divisor;
    M.bg_density = background_density;
    M.n_hist = (double)g->n_histories;
    M.n_batches_minus_1 = (double)(g->n_batches - 1);
    M.rel_defined = (g->n_batches >= 2 && g->n_histories > 0) ? 1 : 0;
    M.n_prims = n_prims;
    const long long nv = g->k.nvox;
    double* out[4] = {dose_Gy, h10_pSv, kerma_rel, h10_rel};
    double* dev[4] = {dose_Gy, h10_pSv, kerma_rel, h10_rel};
    if (!on_device) {
        if (!g->d_maps) CC_CUDA(cudaMalloc(&g->d_maps, (size_t)4 * nv * sizeof(double)));
        for (int j = 0; j < 4; ++j) dev[j] = out[j] ? g->d_maps + (size_t)j * nv : nullptr;
    }
    MapPrim* d_prims = nullptr;
    if (n_prims > 0) {
        CC_CUDA(cudaMalloc(&d_prims, mp.size() * sizeof(MapPrim)));
        cudaError_t e = cudaMemcpyAsync(d_prims, mp.data(), mp.size() * sizeof(MapPrim), cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) { cudaFree(d_prims); return set_error(CC_E_DEVICE, cudaGetErrorString(e)); }
    }
    const int threads = 256;
    const int blocks = std::max(1, std::min((int)((nv + threads - 1) / threads), c->sm_count * 8));
    // totals as cc_grid_download gives them: folded batches plus the pending one
    maps_kernel<<<blocks, threads, 0, c->stream>>>((const double2*)g->d_total, (const double2*)g->d_scratch,
                                                   (const double2*)g->d_q, d_prims, M, dev[0], dev[1], dev[2], dev[3]);
    cudaError_t e = cudaGetLastError();
    for (int j = 0; j < 4 && e == cudaSuccess && !on_device; ++j)
        if (out[j]) e = cudaMemcpyAsync(out[j], dev[j], (size_t)nv * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_prims);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("grid maps: ") + cudaGetErrorString(e));
    return CC_OK;
}

int cc_grid_end_batch(cc_grid* g, int64_t n_hist) {
    if (!g) return set_error(CC_E_INVALID, "grid is NULL");
    if (!(g->flags & CC_GRID_STATS) || n_hist <= 0) return CC_OK;
    long long cnt = n_hist;
    int rc = fold_batches(g, 1, &cnt, 0);              // the pending batch is in FP64 cells
    if (rc != CC_OK) return rc;
    CC_CUDA(cudaStreamSynchronize(g->ctx->stream));
    return CC_OK;
}

int cc_grid_download(cc_grid* g, double* kerma, double* h10, double* k2, double* h2, int32_t* nhit,
                     int64_t* n_batches, int64_t* n_histories) {
    if (!g) return set_error(CC_E_INVALID, "grid is NULL");
    cc_ctx* c = g->ctx;
    CC_CUDA(cudaSetDevice(c->device));
    const long long nv = g->k.nvox;
    const bool stats = g->d_q != nullptr;
    const size_t bytes = (size_t)nv * ((stats ? 4 : 2) * sizeof(double) + (stats ? sizeof(int) : 0));
    // device staging allocated on the first download and kept with the grid
    if (!g->d_out) CC_CUDA(cudaMalloc(&g->d_out, bytes));
    double* ok = (double*)g->d_out;
    double* oh = ok + nv;
    double* ok2 = stats ? oh + nv : nullptr;
    double* oh2 = stats ? ok2 + nv : nullptr;
    int* on = stats ? (int*)(oh2 + nv) : nullptr;
    int threads = 256;
    int blocks = std::max(1, std::min((int)((nv + threads - 1) / threads), c->sm_count * 8));
    unpack_kernel<<<blocks, threads, 0, c->stream>>>((const double2*)g->d_total, (const double2*)g->d_scratch,
                                                     (const double2*)g->d_q, g->d_nhit, ok, oh, ok2, oh2, on, nv);
    CC_CUDA(cudaGetLastError());
    // each output goes straight into the caller's array when that is
    // page-locked host memory, else through the grid's pinned staging
    const size_t b8 = (size_t)nv * sizeof(double);
    struct Out { void* dst; const char* src; size_t bytes; bool pinned; };
    Out outs[5] = {{kerma, (const char*)ok, b8, false}, {h10, (const char*)oh, b8, false},
                   {stats ? k2 : nullptr, (const char*)ok2, b8, false}, {stats ? h2 : nullptr, (const char*)oh2, b8, false},
                   {stats ? nhit : nullptr, (const char*)on, (size_t)nv * sizeof(int), false}};
    bool staged = false;
    for (Out& o : outs) {
        if (!o.dst) continue;
        cudaPointerAttributes at;
        o.pinned = cudaPointerGetAttributes(&at, o.dst) == cudaSuccess && at.type == cudaMemoryTypeHost;
        cudaGetLastError();
        // pinned host staging, allocated when an output first needs it
        if (!o.pinned && !g->h_out && cudaHostAlloc((void**)&g->h_out, bytes, cudaHostAllocDefault) != cudaSuccess) {
            g->h_out = nullptr;
            cudaStreamSynchronize(c->stream);     // copies already queued finish before the error returns
            return set_error(CC_E_NOMEM, "pinned host staging for the grid download failed");
        }
        const size_t off = (size_t)(o.src - g->d_out);
        if (o.pinned) {
            CC_CUDA(cudaMemcpyAsync(o.dst, o.src, o.bytes, cudaMemcpyDeviceToHost, c->stream));
        } else {
            CC_CUDA(cudaMemcpyAsync(g->h_out + off, o.src, o.bytes, cudaMemcpyDeviceToHost, c->stream));
            staged = true;
        }
    }
    CC_CUDA(cudaStreamSynchronize(c->stream));
    if (staged)
        for (const Out& o : outs)
            if (o.dst && !o.pinned) memcpy(o.dst, g->h_out + (size_t)(o.src - g->d_out), o.bytes);
    if (n_batches) *n_batches = g->n_batches;
    if (n_histories) *n_histories = g->n_histories;
    return CC_OK;
}

// ---------------------------------------------------------------------------

static int status_to_error(unsigned st) {
    if (st & ST_ENERGY) return set_error(CC_E_ENERGY_RANGE, "photon energy left the cross-section table range [1, 150] keV");
    if (st & ST_RAYLEIGH_Q) return set_error(CC_E_RAYLEIGH_Q_RANGE, "q(E) beyond the Rayleigh form-factor table");
    if (st & ST_STEPS) return set_error(CC_E_TIMEOUT, "a photon exceeded the step limit");
    if (st & ST_BOUNDS) return set_error(CC_E_BOUNDS, "an index check failed inside the kernel");
    return CC_OK;
}

// Blocks per SM of a launch whose grid's scratch slot exceeds
// SLOT_BYTES_COMPACT, unless the context sets its own: fewer histories in
// flight span fewer batch slots, whose scattered reductions then hit L2
// more often.  Measured on the CT workload (246 MB slots, batches of
// 200,000 histories): 2.89e8 histories/s with 1 block of 256 per SM, 2.68e8
// with 2, 2.52e8 with 3, 2.46e8 with 4.
constexpr int BIG_GRID_BLOCKS_PER_SM = 1;

static int grid_blocks_for(cc_ctx* c, size_t smem, bool fs, bool tl, bool big_grid) {
    int per_sm = c->blocks_per_sm;
    if (per_sm == 0) {
        int occ = 0;
        cudaError_t e;
        if (fs && tl) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, transport_kernel<true, true>, c->block, smem);
        else if (fs) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, transport_kernel<true, false>, c->block, smem);
        else if (tl) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, transport_kernel<false, true>, c->block, smem);
        else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, transport_kernel<false, false>, c->block, smem);
        if (e != cudaSuccess || occ < 1) occ = 1;
        per_sm = big_grid ? std::min(occ, BIG_GRID_BLOCKS_PER_SM) : occ;
    }
    return c->sm_count * per_sm;
}

// Page-locked records and events of the launch ring, created on first use.
static int ensure_ring(cc_ctx* c) {
    if (c->h_ring) return CC_OK;
    const size_t per = (size_t)MAX_SCRATCH * MAX_MATS * sizeof(double) + 10 * sizeof(unsigned long long);
    char* h = nullptr;
    if (cudaHostAlloc((void**)&h, per * cc_ctx::LAUNCH_RING, cudaHostAllocDefault) != cudaSuccess)
        return set_error(CC_E_NOMEM, "page-locked launch records");
    for (int i = 0; i < cc_ctx::LAUNCH_RING; ++i) {
        auto& r = c->ring[i];
        r.h_edep = (double*)(h + per * i);
        r.h_cnt = (unsigned long long*)(h + per * i + (size_t)MAX_SCRATCH * MAX_MATS * sizeof(double));
        r.h_status = (unsigned*)(r.h_cnt + 8);
        if (cudaEventCreate(&r.k0) != cudaSuccess || cudaEventCreate(&r.k1) != cudaSuccess ||
            cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming) != cudaSuccess) {
            cudaFreeHost(h);
            return set_error(CC_E_DEVICE, "launch ring events");
        }
    }
    c->h_ring = h;
    return CC_OK;
}

// One launch of the transport kernel plus the copies of its reductions into
// a ring record, queued on the context's stream without waiting.
static int enqueue_launch(cc_ctx* c, const cc_scene* scene, const cc_tables* tables, const KSource* src,
                          cc_grid* grid, double* tally_base, int n_slots, long long batch_size, KRun R,
                          int cell32, cc_ctx::LaunchRec& rec) {
    const KTables& T = tables->k;
    R.n_scratch = n_slots;
    R.batch_size = batch_size;
    const bool big_grid = grid && (size_t)grid->k.nvox * 16 > SLOT_BYTES_COMPACT;
    R.chunk = big_grid ? HIST_CHUNK_COMPACT : HIST_CHUNK_SPREAD;
    R.max_steps = c->max_steps;
    R.status = c->d_status;
    R.counters = c->d_counters;
    R.work = c->d_counters + 6;
    size_t n_acc = (size_t)n_slots * T.n_mat;
    if (n_acc > (size_t)MAX_SCRATCH * MAX_MATS) return set_error(CC_E_INVALID, "too many batches x materials per launch");
    cudaStream_t st = c->stream;
    CC_CUDA(cudaMemsetAsync(c->d_edep, 0, n_acc * sizeof(double), st));
    CC_CUDA(cudaMemsetAsync(c->d_counters, 0, 8 * sizeof(unsigned long long), st));
    CC_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), st));
    R.edep = c->d_edep;
    KGrid G;
    memset(&G, 0, sizeof(G));
    bool tl = grid != nullptr;
    if (tl) { G = grid->k; G.tally = tally_base; G.tally32 = cell32; }
    KSource S;
    memset(&S, 0, sizeof(S));
    bool fs = src != nullptr;
    if (fs) S = *src;
    size_t smem = n_acc * sizeof(double);
    int blocks = grid_blocks_for(c, smem, fs, tl, big_grid);
    const bool defer = tl && c->tally_queue;
    R.defer = defer ? 1 : 0;
    if (defer) {
        long long want = std::max<long long>(1LL << 20, (long long)(c->seg_per_history * (double)R.n) + 1024);
        want = std::min<long long>(want, (long long)(SEG_QUEUE_MAX_BYTES / sizeof(SegRec)));
        if (c->tally_queue_cap > 0) want = c->tally_queue_cap;
        if (want > c->seg_alloc || (c->tally_queue_cap > 0 && want != c->seg_alloc)) {
            // grow-only; launches still queued may read the old queue
            CC_CUDA(cudaStreamSynchronize(st));
            cudaFree(c->d_seg);
            c->d_seg = nullptr;
            c->seg_alloc = 0;
            if (cudaMalloc(&c->d_seg, (size_t)want * sizeof(SegRec)) != cudaSuccess)
                return set_error(CC_E_NOMEM, "device allocation of the tally's segment queue failed");
            c->seg_alloc = want;
        }
        R.seg = c->d_seg;
        R.seg_cap = c->seg_alloc;
    }
    CC_CUDA(cudaEventRecord(rec.k0, st));
    cudaError_t e;
    const bool heel = fs && S.heel_n > 0;
    if (fs && tl && heel) e = launch_transport<true, true, true>(c, T, scene->k, G, S, R, smem, blocks);
    else if (fs && heel) e = launch_transport<true, false, true>(c, T, scene->k, G, S, R, smem, blocks);
    else if (fs && tl) e = launch_transport<true, true>(c, T, scene->k, G, S, R, smem, blocks);
    else if (fs) e = launch_transport<true, false>(c, T, scene->k, G, S, R, smem, blocks);
    else if (tl) e = launch_transport<false, true>(c, T, scene->k, G, S, R, smem, blocks);
    else e = launch_transport<false, false>(c, T, scene->k, G, S, R, smem, blocks);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("transport launch: ") + cudaGetErrorString(e));
    if (defer) {
        tally_kernel<<<c->sm_count * c->tally_blocks_per_sm, BLOCK, 0, st>>>(G, R.seg, R.counters + 7, R.seg_cap,
                                                                          R.counters);
        e = cudaGetLastError();
        if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("tally launch: ") + cudaGetErrorString(e));
    }
    CC_CUDA(cudaEventRecord(rec.k1, st));
    e = cudaMemcpyAsync(rec.h_edep, c->d_edep, n_acc * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rec.h_cnt, c->d_counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rec.h_status, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(rec.done, st);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("transport: ") + cudaGetErrorString(e));
    rec.ns = n_slots;
    rec.seg_cap = defer ? R.seg_cap : 0;
    rec.busy = true;
    return CC_OK;
}

// Waits for a ring record's launch (its copies were queued after the kernel)
// and returns its status as an error code.
static int finish_launch(cc_ctx* c, cc_ctx::LaunchRec& rec, float* kernel_ms) {
    cudaError_t e = cudaEventSynchronize(rec.done);
    rec.busy = false;
    // a launch that offered its queue more segments than it held: provide
    // for a quarter more per history from the next launch on
    if (e == cudaSuccess && rec.n > 0 && (long long)rec.h_cnt[7] > rec.seg_cap)
        c->seg_per_history = std::max(c->seg_per_history, 1.25 * (double)rec.h_cnt[7] / (double)rec.n);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("transport: ") + cudaGetErrorString(e));
    if (kernel_ms) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, rec.k0, rec.k1);
        *kernel_ms = ms;
    }
    return status_to_error(*rec.h_status);
}

// One synchronous launch: queued, then waited for.
static int run_launch(cc_ctx* c, const cc_scene* scene, const cc_tables* tables, const KSource* src,
                      cc_grid* grid, double* tally_base, int n_slots, long long batch_size,
                      KRun R, std::vector<double>& edep_slots, unsigned long long* counters_out,
                      float* kernel_ms, int cell32 = 0) {
    int rc = ensure_ring(c);
    if (rc != CC_OK) return rc;
    cc_ctx::LaunchRec& rec = c->ring[0];
    rc = enqueue_launch(c, scene, tables, src, grid, tally_base, n_slots, batch_size, R, cell32, rec);
    if (rc != CC_OK) return rc;
    rec.n = R.n;
    rc = finish_launch(c, rec, kernel_ms);
    const size_t n_acc = (size_t)n_slots * tables->k.n_mat;
    edep_slots.assign(rec.h_edep, rec.h_edep + n_acc);
    for (int k = 0; k < 6; ++k) counters_out[k] = rec.h_cnt[k];
    return rc;
}

static int transport_common(cc_ctx* c, const cc_scene* scene, const cc_tables* tables, cc_grid* grid,
                            int64_t n, double* d_pos, double* d_dir, double* d_en, uint64_t seed,
                            uint64_t stream_offset, int32_t fluorescence, int32_t* d_nsc,
                            uint8_t* d_abs, uint8_t* d_esc, double* edep, int64_t* n_fluor) {
    KRun R;
    memset(&R, 0, sizeof(R));
    R.n = n;
    R.first = (long long)stream_offset;
    R.fluorescence = fluorescence;
    R.seed = seed;
    R.pos = d_pos; R.dir = d_dir; R.energy = d_en;
    R.n_scatter = d_nsc; R.absorbed = d_abs; R.escaped = d_esc;
    // a statistics grid's slot 0 is its pending batch (FP64 cells, folded by
    // cc_grid_end_batch); any other grid's slot 0 is folded after the call
    double* tally = grid ? grid->d_scratch : nullptr;
    const bool pending = grid && (grid->flags & CC_GRID_STATS);
    const int cell32 = (grid && !pending) ? cell32_for(c, n) : 0;
    std::vector<double> slots;
    unsigned long long cnt[6] = {0, 0, 0, 0, 0, 0};
    int rc = run_launch(c, scene, tables, nullptr, grid, tally, 1, std::max<long long>(n, 1), R, slots, cnt, nullptr,
                        cell32);
    if (rc != CC_OK) return rc;
    if (grid && !pending) {
        rc = fold_plain(grid, 1, cell32);
        if (rc != CC_OK) return rc;
    }
    if (edep) for (int m = 0; m < tables->n_mat; ++m) edep[m] += slots[m];
    if (n_fluor) *n_fluor = (int64_t)cnt[3];
    return CC_OK;
}

int cc_transport_photons_device(cc_ctx* c, const cc_scene* scene, const cc_tables* tables, cc_grid* grid,
                                int64_t n, double* d_pos, double* d_dir, double* d_en, uint64_t seed,
                                uint64_t stream_offset, int32_t fluorescence, int32_t* d_nsc,
                                uint8_t* d_abs, uint8_t* d_esc, double* edep, int64_t* n_fluor) {
    if (!c || !scene || !tables) return set_error(CC_E_INVALID, "NULL argument");
    if (n < 0) return set_error(CC_E_INVALID, "n < 0");
    if (n == 0) { if (n_fluor) *n_fluor = 0; return CC_OK; }
    if (!d_pos || !d_dir || !d_en) return set_error(CC_E_INVALID, "photon arrays are NULL");
    if (scene->ctx->device != c->device || tables->ctx->device != c->device ||
        (grid && grid->ctx->device != c->device))
        return set_error(CC_E_INVALID, "scene, tables and grid must belong to the context's device");
    CC_CUDA(cudaSetDevice(c->device));
    return transport_common(c, scene, tables, grid, n, d_pos, d_dir, d_en, seed, stream_offset,
                            fluorescence, d_nsc, d_abs, d_esc, edep, n_fluor);
}

// Interaction counts widened to int64 for the host (the reference's dtype).
__global__ void widen_kernel(const int32_t* __restrict__ in, int64_t* __restrict__ out, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = in[i];
}

// Photon counts from which cc_transport_photons overlaps its copies with
// the transport: the photons go in LAUNCH_RING chunks, each uploaded on one
// copy stream, transported, and downloaded on another while the next chunk
// runs.  Histories stay keyed by their index, so the results are those of
// one launch over all photons.
constexpr long long PIPE_MIN_PHOTONS = 1LL << 21;

static int ensure_copy_streams(cc_ctx* c) {
    if (c->s_in) return CC_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking);
    for (int i = 0; i < cc_ctx::LAUNCH_RING && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_k[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("copy streams: ") + cudaGetErrorString(e));
    return CC_OK;
}

static int transport_photons_chunked(cc_ctx* c, const cc_scene* scene, const cc_tables* tables, cc_grid* grid,
                                     int64_t n, double* pos, double* dir, double* energy, uint64_t seed,
                                     uint64_t stream_offset, int32_t fluorescence, int64_t* n_scatter,
                                     uint8_t* absorbed, uint8_t* escaped, double* edep, int64_t* n_fluor,
                                     double* d_pos, double* d_dir, double* d_en, int64_t* d_nsc64, int32_t* d_nsc,
                                     uint8_t* d_abs, uint8_t* d_esc) {
    int rc = ensure_ring(c);
    if (rc == CC_OK) rc = ensure_copy_streams(c);
    if (rc != CC_OK) return rc;
    const int K = cc_ctx::LAUNCH_RING;
    const long long per = (n + K - 1) / K;
    cudaStream_t st = c->stream;
    // as transport_common: a statistics grid's slot 0 is its pending batch,
    // any other grid's slot 0 is folded after the call
    double* tally = grid ? grid->d_scratch : nullptr;
    const bool pending = grid && (grid->flags & CC_GRID_STATS);
    const int cell32 = (grid && !pending) ? cell32_for(c, n) : 0;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < K && e == cudaSuccess; ++i) {
        const long long a = std::min<long long>(n, i * per), m = std::min<long long>(n, a + per) - a;
        if (m <= 0) break;
        e = cudaMemcpyAsync(d_pos + 3 * a, pos + 3 * a, (size_t)m * 3 * sizeof(double), cudaMemcpyHostToDevice, c->s_in);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_dir + 3 * a, dir + 3 * a, (size_t)m * 3 * sizeof(double), cudaMemcpyHostToDevice, c->s_in);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_en + a, energy + a, (size_t)m * sizeof(double), cudaMemcpyHostToDevice, c->s_in);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_in[i], c->s_in);
    }
    int used = 0;
    for (int i = 0; i < K && e == cudaSuccess && rc == CC_OK; ++i) {
        const long long a = std::min<long long>(n, i * per), m = std::min<long long>(n, a + per) - a;
        if (m <= 0) break;
        e = cudaStreamWaitEvent(st, c->ev_in[i], 0);
        if (e != cudaSuccess) break;
        KRun R;
        memset(&R, 0, sizeof(R));
        R.n = m;
        R.first = (long long)stream_offset + a;
        R.fluorescence = fluorescence;
        R.seed = seed;
        R.pos = d_pos + 3 * a; R.dir = d_dir + 3 * a; R.energy = d_en + a;
        R.n_scatter = n_scatter ? d_nsc + a : nullptr;
        R.absorbed = absorbed ? d_abs + a : nullptr;
        R.escaped = escaped ? d_esc + a : nullptr;
        rc = enqueue_launch(c, scene, tables, nullptr, grid, tally, 1, m, R, cell32, c->ring[i]);
        if (rc != CC_OK) break;
        c->ring[i].n = m;
        ++used;
        if (n_scatter) {
            const int blocks = (int)std::max<long long>(1, std::min<long long>((m + 255) / 256, (long long)c->sm_count * 8));
            widen_kernel<<<blocks, 256, 0, st>>>(d_nsc + a, d_nsc64 + a, m);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_k[i], st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_out, c->ev_k[i], 0);
        cudaStream_t so = c->s_out;
        if (e == cudaSuccess) e = cudaMemcpyAsync(pos + 3 * a, d_pos + 3 * a, (size_t)m * 3 * sizeof(double), cudaMemcpyDeviceToHost, so);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dir + 3 * a, d_dir + 3 * a, (size_t)m * 3 * sizeof(double), cudaMemcpyDeviceToHost, so);
        if (e == cudaSuccess) e = cudaMemcpyAsync(energy + a, d_en + a, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, so);
        if (e == cudaSuccess && n_scatter) e = cudaMemcpyAsync(n_scatter + a, d_nsc64 + a, (size_t)m * sizeof(int64_t), cudaMemcpyDeviceToHost, so);
        if (e == cudaSuccess && absorbed) e = cudaMemcpyAsync(absorbed + a, d_abs + a, (size_t)m, cudaMemcpyDeviceToHost, so);
        if (e == cudaSuccess && escaped) e = cudaMemcpyAsync(escaped + a, d_esc + a, (size_t)m, cudaMemcpyDeviceToHost, so);
    }
    if (e == cudaSuccess && rc == CC_OK && grid && !pending) rc = fold_plain(grid, 1, cell32);
    // the chunks' reductions, in launch order
    unsigned long long fl = 0;
    for (int i = 0; i < used; ++i) {
        const int frc = finish_launch(c, c->ring[i], nullptr);
        if (rc == CC_OK) rc = frc;
        if (edep) for (int m = 0; m < tables->n_mat; ++m) edep[m] += c->ring[i].h_edep[m];
        fl += c->ring[i].h_cnt[3];
    }
    cudaError_t e2 = cudaStreamSynchronize(c->s_out);
    cudaError_t e3 = cudaStreamSynchronize(st);
    cudaError_t e4 = cudaStreamSynchronize(c->s_in);
    if (e == cudaSuccess) e = e2 != cudaSuccess ? e2 : (e3 != cudaSuccess ? e3 : e4);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("chunked transport: ") + cudaGetErrorString(e));
    if (rc == CC_OK && n_fluor) *n_fluor = (int64_t)fl;
    return rc;
}

int cc_transport_photons(cc_ctx* c, const cc_scene* scene, const cc_tables* tables, cc_grid* grid,
                         int64_t n, double* pos, double* dir, double* energy, uint64_t seed,
                         uint64_t stream_offset, int32_t fluorescence, int64_t* n_scatter,
                         uint8_t* absorbed, uint8_t* escaped, double* edep, int64_t* n_fluor) {
    if (!c || !scene || !tables) return set_error(CC_E_INVALID, "NULL argument");
    if (n < 0) return set_error(CC_E_INVALID, "n < 0");
    if (n == 0) { if (n_fluor) *n_fluor = 0; return CC_OK; }
    if (!pos || !dir || !energy) return set_error(CC_E_INVALID, "photon arrays are NULL");
    CC_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    size_t b3 = (size_t)n * 3 * sizeof(double), b1 = (size_t)n * sizeof(double);
    size_t total = 2 * b3 + b1 + (size_t)n * (sizeof(int64_t) + sizeof(int32_t) + 2);
    if (total > c->io_bytes) {
        cudaFree(c->d_io);
        c->d_io = nullptr;
        c->io_bytes = 0;
        CC_CUDA(cudaMalloc(&c->d_io, total));
        c->io_bytes = total;
    }
    char* buf = c->d_io;
    double* d_pos = (double*)buf;
    double* d_dir = (double*)(buf + b3);
    double* d_en = (double*)(buf + 2 * b3);
    int64_t* d_nsc64 = (int64_t*)(buf + 2 * b3 + b1);
    int32_t* d_nsc = (int32_t*)(d_nsc64 + n);
    uint8_t* d_abs = (uint8_t*)(d_nsc + n);
    uint8_t* d_esc = d_abs + n;
    if (n >= PIPE_MIN_PHOTONS)
        return transport_photons_chunked(c, scene, tables, grid, n, pos, dir, energy, seed, stream_offset,
                                         fluorescence, n_scatter, absorbed, escaped, edep, n_fluor, d_pos, d_dir,
                                         d_en, d_nsc64, d_nsc, d_abs, d_esc);
    cudaError_t e = cudaMemcpyAsync(d_pos, pos, b3, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_dir, dir, b3, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_en, energy, b1, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("upload: ") + cudaGetErrorString(e));
    int rc = transport_common(c, scene, tables, grid, n, d_pos, d_dir, d_en, seed, stream_offset,
                              fluorescence, n_scatter ? d_nsc : nullptr, absorbed ? d_abs : nullptr,
                              escaped ? d_esc : nullptr, edep, n_fluor);
    if (rc == CC_OK) {
        e = cudaMemcpyAsync(pos, d_pos, b3, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dir, d_dir, b3, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(energy, d_en, b1, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && n_scatter) {
            const int blocks = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)c->sm_count * 8));
            widen_kernel<<<blocks, 256, 0, st>>>(d_nsc, d_nsc64, n);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaMemcpyAsync(n_scatter, d_nsc64, (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess && absorbed) e = cudaMemcpyAsync(absorbed, d_abs, (size_t)n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && escaped) e = cudaMemcpyAsync(escaped, d_esc, (size_t)n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = set_error(CC_E_DEVICE, std::string("download: ") + cudaGetErrorString(e));
    }
    return rc;
}

int cc_run(cc_ctx* c, const cc_scene* scene, const cc_tables* tables, const cc_source* src, cc_grid* grid,
           int64_t n_hist, int64_t batch_size, uint64_t seed, int64_t first_history, int32_t fluorescence,
           double* edep, double* edep_sum2, cc_run_out* out) {
    if (!c || !scene || !tables || !src) return set_error(CC_E_INVALID, "NULL argument");
    if (n_hist < 0 || batch_size <= 0) return set_error(CC_E_INVALID, "n_histories < 0 or batch_size <= 0");
    CC_CUDA(cudaSetDevice(c->device));
    const int n_mat = tables->n_mat;
    bool stats = grid && (grid->flags & CC_GRID_STATS);
    // batches per launch: enough histories per launch to hide the tail of
    // the longest histories, bounded by the scratch memory
    long long per_launch_target = 1LL << 22;
    int slots = (int)std::min<long long>(MAX_SCRATCH, std::max<long long>(1, per_launch_target / batch_size));
    slots = std::min(slots, std::max(1, (int)((48 * 1024) / (sizeof(double) * n_mat))));
    // a grid scores every batch into its own scratch slot (the batch
    // statistics need that, and FP32 cells must not sum more than a batch)
    const bool slotted = grid != nullptr;
    const int cell32 = slotted ? cell32_for(c, batch_size) : 0;
    if (grid) {
        size_t per = (size_t)grid->k.nvox * 2 * sizeof(double);
        size_t budget = (size_t)8 << 30;
        slots = (int)std::max<size_t>(1, std::min<size_t>(slots, budget / per));
        int rc = grid_alloc_scratch(grid, slots);
        if (rc != CC_OK) return rc;
    }
    long long done = 0;
    long long launches = 0;
    unsigned long long tot[6] = {0, 0, 0, 0, 0, 0};
    float ms_total = 0.0f;
    double ms_transport = 0.0;
    long long transport_launches = 0;
    int rc = ensure_ring(c);
    if (rc != CC_OK) return rc;
    // Launches are queued up to LAUNCH_RING deep; a launch's reductions are
    // read from its ring record when the record is needed again or at the
    // end, so the host never leaves the GPU idle between launches.  Records
    // are finished in launch order, so the per-batch sums below are added in
    // the same order as with one launch at a time.
    auto finish = [&](cc_ctx::LaunchRec& rec) -> int {
        float kms = 0.f;
        const int frc = finish_launch(c, rec, &kms);
        ms_transport += kms;
        // per-batch collision-estimator moments (ScalarMoments.add_batch, tally.py:204-213)
        for (int b = 0; b < rec.ns; ++b) {
            long long nb = std::min<long long>(batch_size, rec.n - (long long)b * batch_size);
            for (int m = 0; m < n_mat; ++m) {
                double v = rec.h_edep[(size_t)b * n_mat + m];
                if (edep) edep[m] += v;
                if (edep_sum2 && stats) edep_sum2[m] += v * v / (double)nb;
            }
        }
        for (int k = 0; k < 6; ++k) tot[k] += rec.h_cnt[k];
        return frc;
    };
    auto drain = [&](int from) -> int {
        int first_err = CC_OK;
        for (int i = 0; i < cc_ctx::LAUNCH_RING; ++i) {
            cc_ctx::LaunchRec& r = c->ring[(from + i) % cc_ctx::LAUNCH_RING];
            if (!r.busy) continue;
            const int frc = finish(r);
            if (first_err == CC_OK) first_err = frc;
        }
        return first_err;
    };
    CC_CUDA(cudaEventRecord(c->ev0, c->stream));
    long long li = 0;
    while (done < n_hist) {
        int ns = slots;
        long long n_launch = std::min<long long>(n_hist - done, (long long)ns * batch_size);
        ns = (int)((n_launch + batch_size - 1) / batch_size);
        KRun R;
        memset(&R, 0, sizeof(R));
        R.n = n_launch;
        R.first = first_history + done;
        R.fluorescence = fluorescence;
        R.seed = seed;
        double* tally = grid ? grid->d_scratch : nullptr;
        const int ri = (int)(li % cc_ctx::LAUNCH_RING);
        cc_ctx::LaunchRec& rec = c->ring[ri];
        if (rec.busy) {
            rc = finish(rec);
            if (rc != CC_OK) { drain(ri + 1); return rc; }
        }
        rc = enqueue_launch(c, scene, tables, &src->k, grid, tally, slotted ? ns : 1,
                            slotted ? batch_size : std::max<long long>(n_launch, 1), R, cell32, rec);
        if (rc != CC_OK) { drain(ri + 1); cudaStreamSynchronize(c->stream); return rc; }
        rec.n = n_launch;     // rec.ns: its batches (one slot for all histories without a grid)
        ++li;
        ++launches;
        ++transport_launches;
        if (stats) {
            std::vector<long long> counts(ns);
            for (int b = 0; b < ns; ++b) counts[b] = std::min<long long>(batch_size, n_launch - (long long)b * batch_size);
            rc = fold_batches(grid, ns, counts.data(), cell32);
            if (rc != CC_OK) { drain(ri + 1); return rc; }
            launches += ns > 1 ? 1 : ns;
        } else if (grid) {
            rc = fold_plain(grid, ns, cell32);
            if (rc != CC_OK) { drain(ri + 1); return rc; }
            launches += ns > 1 ? 1 : ns;
        }
        done += n_launch;
    }
    CC_CUDA(cudaEventRecord(c->ev1, c->stream));
    rc = drain((int)(li % cc_ctx::LAUNCH_RING));
    CC_CUDA(cudaEventSynchronize(c->ev1));
    cudaEventElapsedTime(&ms_total, c->ev0, c->ev1);
    if (rc != CC_OK) return rc;
    if (out) {
        out->n_histories = n_hist;
        out->n_absorbed = (int64_t)tot[0];
        out->n_escaped = (int64_t)tot[1];
        out->scatter_sum = (int64_t)tot[2];
        out->n_fluorescence = (int64_t)tot[3];
        out->n_batches = (n_hist + batch_size - 1) / batch_size;
        out->gpu_launches = launches;
        out->elapsed_ms = ms_total;
        out->n_steps = (int64_t)tot[4];
        out->n_voxel_visits = (int64_t)tot[5];
        out->transport_ms = ms_transport;
        out->transport_launches = transport_launches;
    }
    return CC_OK;
}

int cc_sample_source(cc_ctx* c, const cc_source* src, int64_t n, uint64_t seed, int64_t first,
                     double* pos, double* dir, double* energy) {
    if (!c || !src || !pos || !dir || !energy) return set_error(CC_E_INVALID, "NULL argument");
    if (n <= 0) return CC_OK;
    CC_CUDA(cudaSetDevice(c->device));
    double* buf = nullptr;
    CC_CUDA(cudaMalloc(&buf, (size_t)n * 7 * sizeof(double)));
    int threads = 256;
    long long blocks = (n + threads - 1) / threads;
    sample_source_kernel<<<(unsigned)blocks, threads, 0, c->stream>>>(src->k, n, first, seed, buf, buf + 3 * n, buf + 6 * n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(pos, buf, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dir, buf + 3 * n, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(energy, buf + 6 * n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("sample_source: ") + cudaGetErrorString(e));
    return CC_OK;
}

int cc_sample_interactions(cc_ctx* c, const cc_tables* tables, int32_t kind, int64_t n, const int32_t* material,
                           const double* energy, uint64_t seed, int32_t fluorescence, double* out_a,
                           double* out_b, int32_t* out_z) {
    if (!c || !tables || !material || !energy || !out_a || !out_b || !out_z)
        return set_error(CC_E_INVALID, "NULL argument");
    if (kind < INTERACT_PHOTO || kind > INTERACT_RAYLEIGH) return set_error(CC_E_INVALID, "unknown interaction kind");
    if (n < 0) return set_error(CC_E_INVALID, "n < 0");
    if (n == 0) return CC_OK;
    if (tables->ctx->device != c->device) return set_error(CC_E_INVALID, "tables belong to another device");
    CC_CUDA(cudaSetDevice(c->device));
    std::vector<phys> ef((size_t)n);
    for (int64_t i = 0; i < n; ++i) ef[i] = (phys)energy[i];
    // [status 256 B][mat n x 4][energy n x 8][z n x 4][a n x 8][b n x 8], sub-arrays 256-byte aligned
    const size_t n4 = ((size_t)n * 4 + 255) / 256 * 256, n8 = ((size_t)n * 8 + 255) / 256 * 256;
    const size_t bytes = 256 + 2 * n4 + 3 * n8;
    char* buf = nullptr;
    CC_CUDA(cudaMalloc(&buf, bytes));
    unsigned* d_st = (unsigned*)buf;
    int* d_mat = (int*)(buf + 256);
    phys* d_e = (phys*)(buf + 256 + n4);
    int* d_z = (int*)(buf + 256 + n4 + n8);
    double* d_a = (double*)(buf + 256 + 2 * n4 + n8);
    double* d_b = d_a + n;
    unsigned st = 0;
    cudaStream_t s = c->stream;
    cudaError_t e = cudaMemsetAsync(d_st, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_mat, material, (size_t)n * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_e, ef.data(), (size_t)n * sizeof(phys), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const int threads = 256;
        interaction_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, s>>>(
            tables->k, kind, n, d_mat, d_e, seed, fluorescence, d_a, d_b, d_z, d_st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_a, d_a, (size_t)n * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_b, d_b, (size_t)n * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_z, d_z, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, d_st, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(buf);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("sample_interactions: ") + cudaGetErrorString(e));
    return status_to_error(st);
}

int cc_philox4x32_10(cc_ctx* c, int64_t n, const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    if (!c || !ctr || !key || !out) return set_error(CC_E_INVALID, "NULL argument");
    if (n < 0) return set_error(CC_E_INVALID, "n < 0");
    if (n == 0) return CC_OK;
    CC_CUDA(cudaSetDevice(c->device));
    uint32_t* buf = nullptr;
    CC_CUDA(cudaMalloc(&buf, (size_t)n * 10 * sizeof(uint32_t)));
    cudaStream_t s = c->stream;
    cudaError_t e = cudaMemcpyAsync(buf, ctr, (size_t)n * 16, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf + 4 * n, key, (size_t)n * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        philox_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, buf, buf + 4 * n, buf + 6 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, buf + 6 * n, (size_t)n * 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(buf);
    if (e != cudaSuccess) return set_error(CC_E_DEVICE, std::string("philox: ") + cudaGetErrorString(e));
    return CC_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free transport of device-resident photons.
//
// Some callers cannot let the engine allocate device memory: a host process
// that hands every library a fixed slice of a pre-sized memory pool, a
// real-time pipeline that forbids allocation once it runs (cudaMalloc and
// cudaFree synchronise the device and can stall its other streams), or a
// plug-in whose host application owns all allocations.  For them this entry
// point keeps the per-call scratch -- the reduction counters, the history
// work counter, the status word and the per-material deposited energy -- in
// one file-scope __device__ array instead of the context's buffers.  Every
// GPU that loads this library holds that array (NOALLOC_SCRATCH_WORDS 64-bit
// words, 512 bytes) until the process exits.
// ---------------------------------------------------------------------------

constexpr int NOALLOC_SCRATCH_WORDS = 64;
// word layout: [0, 6) counters, 6 history work counter, 7 status, [8, 8 + MAX_MATS) deposited energy
static_assert(8 + MAX_MATS <= NOALLOC_SCRATCH_WORDS, "scratch too small for the material limit");
static __device__ __align__(256) unsigned long long g_noalloc_scratch[NOALLOC_SCRATCH_WORDS];

static std::mutex g_noalloc_mutex;
static unsigned long long* g_noalloc_addr[64];   // device address of the array, per device ordinal

int cc_transport_photons_device_noalloc(const cc_scene* scene, const cc_tables* tables, int64_t n,
                                        double* d_pos, double* d_dir, double* d_en, uint64_t seed,
                                        uint64_t stream_offset, int32_t fluorescence, int32_t* d_nsc,
                                        uint8_t* d_abs, uint8_t* d_esc, double* edep,
                                        int64_t* n_fluor, void* stream) {
    if (!scene || !tables) return set_error(CC_E_INVALID, "NULL argument");
    if (n < 0) return set_error(CC_E_INVALID, "n < 0");
    if (tables->n_mat > MAX_MATS)
        return set_error(CC_E_INVALID, "the allocation-free entry point handles at most 16 materials "
                                       "(its static scratch holds 16 deposited-energy sums)");
    if (n == 0) { if (n_fluor) *n_fluor = 0; return CC_OK; }
    if (!d_pos || !d_dir || !d_en) return set_error(CC_E_INVALID, "photon arrays are NULL");
    const int dev = tables->ctx->device;
    if (scene->ctx->device != dev) return set_error(CC_E_INVALID, "scene and tables belong to different devices");
    if (dev < 0 || dev >= 64) return set_error(CC_E_INVALID, "device ordinal out of range");
    CC_CUDA(cudaSetDevice(dev));
    unsigned long long* scratch = nullptr;
    {
        // first call on this device: resolve the array's device address with
        // the device current (the host-side symbol is not a device address)
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_addr[dev]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                return set_error(CC_E_DEVICE, std::string("cudaGetSymbolAddress of the scratch array: ") +
                                                  cudaGetErrorString(e));
            g_noalloc_addr[dev] = (unsigned long long*)ptr;
        }
        scratch = g_noalloc_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    // the array keeps the previous call's contents: clear it
    CC_CUDA(cudaMemsetAsync(scratch, 0, NOALLOC_SCRATCH_WORDS * sizeof(unsigned long long), st));
    KRun R;
    memset(&R, 0, sizeof(R));
    R.n = n;
    R.first = (long long)stream_offset;
    R.fluorescence = fluorescence;
    R.seed = seed;
    R.pos = d_pos; R.dir = d_dir; R.energy = d_en;
    R.n_scatter = d_nsc; R.absorbed = d_abs; R.escaped = d_esc;
    R.n_scratch = 1;
    R.batch_size = n;
    R.max_steps = tables->ctx->max_steps;
    R.counters = scratch;
    R.work = scratch + 6;
    R.status = (unsigned*)(scratch + 7);
    R.edep = (double*)(scratch + 8);
    KGrid G;
    memset(&G, 0, sizeof(G));
    KSource S;
    memset(&S, 0, sizeof(S));
    const size_t smem = (size_t)tables->n_mat * sizeof(double);
    int sms = 0, occ = 0;
    CC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, transport_kernel<false, false>, BLOCK, smem) != cudaSuccess ||
        occ < 1)
        occ = 1;
    transport_kernel<false, false><<<sms * occ, BLOCK, smem, st>>>(tables->k, scene->k, G, S, R);
    CC_CUDA(cudaGetLastError());
    unsigned long long words[8 + MAX_MATS];
    CC_CUDA(cudaMemcpyAsync(words, scratch, sizeof(words), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    // a failed call leaves the caller's accumulators as they were
    const int rc = status_to_error((unsigned)words[7]);
    if (rc != CC_OK) return rc;
    if (edep) {
        const double* dep = (const double*)(words + 8);
        for (int m = 0; m < tables->n_mat; ++m) edep[m] += dep[m];
    }
    if (n_fluor) *n_fluor = (int64_t)words[3];
    return CC_OK;
}

// ---------------------------------------------------------------------------
// Batched multi-scene runs: one persistent launch over many scenes, replayed
// from a CUDA graph.
// ---------------------------------------------------------------------------

}  // extern "C"

struct cc_batch {
    cc_ctx* ctx = nullptr;
    const cc_tables* tables = nullptr;
    int n_scenes = 0;
    int slots = 1;
    int chunk = 256;
    bool tally = false;
    std::vector<cc_grid*> grids;
    std::vector<long long> nhist;
    std::vector<std::vector<long long>> slot_counts;
    KBatch kb;
    char* d_mem = nullptr;
    unsigned long long* h_run = nullptr;      // pinned: seed, fluorescence
    unsigned long long* d_counters = nullptr; // [8]: 4 steps, 5 voxel visits, 6 work
    unsigned* d_status = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int blocks = 0;
    long long launches = 0;                   // kernels per replay
};

static void batch_free(cc_batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_mem);
    cudaFreeHost(b->h_run);
    delete b;
}

extern "C" {

int cc_batch_create(cc_ctx* c, const cc_tables* tables, int32_t n_scenes, const cc_scene* const* scenes,
                    const cc_source* const* sources, cc_grid* const* grids, const int64_t* n_histories,
                    int32_t slots, int32_t chunk, cc_batch** out) {
    if (!c || !tables || !scenes || !sources || !n_histories || !out) return set_error(CC_E_INVALID, "NULL argument");
    if (n_scenes < 1 || n_scenes > (1 << 20)) return set_error(CC_E_INVALID, "n_scenes out of range");
    if (slots < 1 || slots > MAX_SCRATCH) return set_error(CC_E_INVALID, "slots must be in [1, 64]");
    if (chunk < 32 || chunk > 4096) return set_error(CC_E_INVALID, "chunk must be in [32, 4096]");
    CC_CUDA(cudaSetDevice(c->device));
    cc_batch* b = new (std::nothrow) cc_batch();
    if (!b) return set_error(CC_E_NOMEM, "out of host memory");
    b->ctx = c;
    b->tables = tables;
    b->n_scenes = n_scenes;
    b->slots = slots;
    b->chunk = chunk;
    b->tally = grids != nullptr;
    bool heel = false;               // some source carries the heel effect
    std::vector<KScene> hs(n_scenes);
    std::vector<KSource> hsrc(n_scenes);
    std::vector<KGrid> hg(n_scenes);
    std::vector<long long> cf(n_scenes + 1, 0);
    b->nhist.resize(n_scenes);
    b->slot_counts.resize(n_scenes);
    for (int i = 0; i < n_scenes; ++i) {
        if (!scenes[i] || !sources[i] || n_histories[i] < 1) { batch_free(b); return set_error(CC_E_INVALID, "scene " + std::to_string(i) + ": NULL handle or no histories"); }
        hs[i] = scenes[i]->k;
        hsrc[i] = sources[i]->k;
        if (hsrc[i].heel_n > 0) heel = true;
        memset(&hg[i], 0, sizeof(KGrid));
        if (b->tally) {
            cc_grid* g = grids[i];
            if (!g) { batch_free(b); return set_error(CC_E_INVALID, "scene " + std::to_string(i) + ": NULL grid"); }
            if (slots > 1 && !(g->flags & CC_GRID_STATS)) { batch_free(b); return set_error(CC_E_INVALID, "batch statistics need CC_GRID_STATS grids"); }
            if (slots > 1) { int rc = grid_alloc_scratch(g, slots); if (rc != CC_OK) { batch_free(b); return rc; } }
            hg[i] = g->k;
            hg[i].tally = g->d_scratch;
            hg[i].tally32 = cell32_for(c, (n_histories[i] + slots - 1) / slots);
            b->grids.push_back(g);
        }
        b->nhist[i] = n_histories[i];
        cf[i + 1] = cf[i] + (n_histories[i] + chunk - 1) / chunk;
        std::vector<long long>& sc = b->slot_counts[i];
        sc.assign(slots, 0);
        // histories li with floor(li * slots / n) == k
        for (int k = 0; k < slots; ++k) {
            long long lo = (k * n_histories[i] + slots - 1) / slots, hi = ((k + 1) * n_histories[i] + slots - 1) / slots;
            sc[k] = hi - lo;
        }
    }
    // one device block for every table of the batch
    // every sub-array starts on a 256-byte boundary (KScene is 4-byte aligned,
    // KSource and KGrid hold 8-byte pointers)
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t o_sc = 0;
    size_t o_src = al(o_sc + sizeof(KScene) * n_scenes);
    size_t o_g = al(o_src + sizeof(KSource) * n_scenes);
    size_t o_cf = al(o_g + sizeof(KGrid) * n_scenes);
    size_t o_nh = al(o_cf + sizeof(long long) * (n_scenes + 1));
    size_t o_cnt = al(o_nh + sizeof(long long) * n_scenes);
    size_t o_run = al(o_cnt + sizeof(unsigned long long) * 4 * n_scenes);
    size_t o_c8 = al(o_run + 2 * sizeof(unsigned long long));
    size_t o_st = o_c8 + 8 * sizeof(unsigned long long);
    size_t total = al(o_st + 16);
    if (cudaMalloc(&b->d_mem, total) != cudaSuccess) { batch_free(b); return set_error(CC_E_NOMEM, "device allocation of the batch failed"); }
    if (cudaHostAlloc((void**)&b->h_run, 2 * sizeof(unsigned long long), cudaHostAllocDefault) != cudaSuccess) {
        batch_free(b);
        return set_error(CC_E_NOMEM, "pinned host allocation failed");
    }
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpy(b->d_mem + o_sc, hs.data(), sizeof(KScene) * n_scenes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_mem + o_src, hsrc.data(), sizeof(KSource) * n_scenes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && b->tally) e = cudaMemcpy(b->d_mem + o_g, hg.data(), sizeof(KGrid) * n_scenes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_mem + o_cf, cf.data(), sizeof(long long) * (n_scenes + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_mem + o_nh, b->nhist.data(), sizeof(long long) * n_scenes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { batch_free(b); return set_error(CC_E_DEVICE, std::string("batch upload: ") + cudaGetErrorString(e)); }
    KBatch& k = b->kb;
    k.scenes = (const KScene*)(b->d_mem + o_sc);
    k.sources = (const KSource*)(b->d_mem + o_src);
    k.grids = (const KGrid*)(b->d_mem + o_g);
    k.chunk_first = (const long long*)(b->d_mem + o_cf);
    k.n_hist = (const long long*)(b->d_mem + o_nh);
    k.scene_cnt = (unsigned long long*)(b->d_mem + o_cnt);
    k.run = (const unsigned long long*)(b->d_mem + o_run);
    k.n_scenes = n_scenes;
    k.chunk = chunk;
    k.slots = slots;
    k.n_chunks = cf[n_scenes];
    b->d_counters = (unsigned long long*)(b->d_mem + o_c8);
    b->d_status = (unsigned*)(b->d_mem + o_st);
    KRun R;
    memset(&R, 0, sizeof(R));
    R.max_steps = c->max_steps;
    R.status = b->d_status;
    R.counters = b->d_counters;
    R.work = b->d_counters + 6;
    // launch shape: the context's block size and blocks per SM (the autotuner sets them)
    int per_sm = c->blocks_per_sm;
    if (per_sm == 0) {
        int occ = 0;
        cudaError_t oe = b->tally ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel<true>, c->block, 0)
                                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel<false>, c->block, 0);
        per_sm = (oe == cudaSuccess && occ > 0) ? occ : 1;
    }
    b->blocks = c->sm_count * per_sm;
    // capture: clear the counters, take the seed, transport, fold the batches
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_mem + o_cnt, 0, sizeof(unsigned long long) * 4 * n_scenes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_mem + o_c8, 0, total - o_c8, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_mem + o_run, b->h_run, 2 * sizeof(unsigned long long), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if (b->tally && heel) batch_kernel<true, true><<<b->blocks, c->block, 0, st>>>(tables->k, k, R);
        else if (b->tally) batch_kernel<true><<<b->blocks, c->block, 0, st>>>(tables->k, k, R);
        else if (heel) batch_kernel<false, true><<<b->blocks, c->block, 0, st>>>(tables->k, k, R);
        else batch_kernel<false><<<b->blocks, c->block, 0, st>>>(tables->k, k, R);
        e = cudaGetLastError();
        b->launches = 1;
    }
    if (e == cudaSuccess && b->tally) {
        int threads = 256;
        for (int i = 0; i < n_scenes && e == cudaSuccess; ++i) {
            cc_grid* g = grids[i];
            const int cell32 = hg[i].tally32;
            int nb = std::max(1, std::min((int)((g->k.nvox + threads - 1) / threads), c->sm_count * 8));
            if (slots > 1) {
                // all batch slots of the scene in one fold
                FoldSlots F;
                memset(&F, 0, sizeof(F));
                F.n = slots;
                for (int sl = 0; sl < slots; ++sl)
                    if (b->slot_counts[i][sl] > 0) F.inv_nb[sl] = 1.0 / (double)b->slot_counts[i][sl];
                fold_slots_kernel<<<nb, threads, 0, st>>>((double2*)g->d_total, (double2*)g->d_q, g->d_nhit,
                                                          (double2*)g->d_scratch, g->k.nvox, F, cell32);
                ++b->launches;
                e = cudaGetLastError();
                continue;
            }
            for (int sl = 0; sl < slots; ++sl) {
                long long cnt = b->slot_counts[i][sl];
                if (cnt <= 0) continue;
                double2* scr = (double2*)(g->d_scratch + (size_t)sl * 2 * g->k.nvox);
                if (slots > 1)
                    fold_kernel<<<nb, threads, 0, st>>>((double2*)g->d_total, (double2*)g->d_q, g->d_nhit, scr,
                                                         g->k.nvox, 1.0 / (double)cnt, cell32);
                else
                    fold_plain_kernel<<<nb, threads, 0, st>>>((double2*)g->d_total, scr, g->k.nvox, cell32);
                ++b->launches;
            }
            e = cudaGetLastError();
        }
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    if (e == cudaSuccess) e = e2;
    b->graph = graph;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
    if (e != cudaSuccess) { batch_free(b); return set_error(CC_E_DEVICE, std::string("batch graph: ") + cudaGetErrorString(e)); }
    *out = b;
    return CC_OK;
}

int cc_batch_run(cc_batch* b, uint64_t seed, int32_t fluorescence, int64_t* scene_counts, cc_run_out* out) {
    if (!b) return set_error(CC_E_INVALID, "batch is NULL");
    cc_ctx* c = b->ctx;
    CC_CUDA(cudaSetDevice(c->device));
    b->h_run[0] = seed;
    b->h_run[1] = (unsigned long long)(fluorescence != 0);
    cudaStream_t st = c->stream;
    CC_CUDA(cudaEventRecord(c->ev0, st));
    CC_CUDA(cudaGraphLaunch(b->exec, st));
    CC_CUDA(cudaEventRecord(c->ev1, st));
    std::vector<unsigned long long> cnt(4 * (size_t)b->n_scenes);
    unsigned long long c8[8];
    unsigned status = 0;
    CC_CUDA(cudaMemcpyAsync(cnt.data(), b->kb.scene_cnt, cnt.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaMemcpyAsync(c8, b->d_counters, sizeof(c8), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaMemcpyAsync(&status, b->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    long long tot = 0;
    for (int i = 0; i < b->n_scenes; ++i) tot += b->nhist[i];
    if (b->tally && b->slots > 1)
        for (int i = 0; i < b->n_scenes; ++i) {
            cc_grid* g = b->grids[i];
            for (int sl = 0; sl < b->slots; ++sl)
                if (b->slot_counts[i][sl] > 0) { g->n_batches += 1; g->n_histories += b->slot_counts[i][sl]; }
        }
    if (scene_counts)
        for (size_t i = 0; i < cnt.size(); ++i) scene_counts[i] = (int64_t)cnt[i];
    if (out) {
        memset(out, 0, sizeof(*out));
        out->n_histories = tot;
        for (int i = 0; i < b->n_scenes; ++i) {
            out->n_absorbed += (int64_t)cnt[4 * i];
            out->n_escaped += (int64_t)cnt[4 * i + 1];
            out->scatter_sum += (int64_t)cnt[4 * i + 2];
            out->n_fluorescence += (int64_t)cnt[4 * i + 3];
        }
        out->n_batches = b->slots;
        out->gpu_launches = b->launches;
        out->elapsed_ms = ms;
        out->n_steps = (int64_t)c8[4];
        out->n_voxel_visits = (int64_t)c8[5];
        out->transport_ms = ms;
        out->transport_launches = 1;
    }
    return status_to_error(status);
}

int cc_batch_destroy(cc_batch* b) {
    if (!b) return CC_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    batch_free(b);
    return CC_OK;
}

}  // extern "C"
