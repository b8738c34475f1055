// Phase 2 kernels: see wg_phase2.cuh for the job structure.
//
// Every floating-point expression keeps the reference's operation order (the library is built
// with -fmad=false, the reference with -ffp-contract=off), so densities, heights and verdicts
// are bit-identical to lysh's.  Reference functions restated here, by file:
//
//   noise.c:200-290          Perlin / octave / DoublePerlin sampling, legacy octave creation
//   interp_noise.c:100-139   the 26.1 blended base noise (old_blended_noise)
//   terrain.c:22-44          terrain info at biome coordinates
//   spline.c:10-131          float spline evaluation, normalized weirdness (1.18 and 26.1)
//   column_top.c:1-130       preliminary surface level and overworld offset
//   density.c:1-281          the non-interpolated density column, noodle children, squeeze
//   phase2.c:44-194,318-456  interpolation grid, density / block / height queries
//   aquifer.c:1-563          computeFluid / computeSubstance (26.1 NoiseBasedAquifer)
//   carver.c:1-523           cave / canyon carvers over a target chunk
//   biome.c:17-156           the biome R-tree search and the swamp-hut biome gate
//   eval.c:41-242            orientation, wet columns, flood short-circuit, verdict
#include <cuda_runtime.h>

#include "wg_phase2.cuh"

namespace wg {
namespace {

// ------------------------------------------------------------------------------------
// Java-semantics helpers (mcmath.h)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double mc_clamp(double v, double lo, double hi) {
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}
__device__ __forceinline__ double mc_lerp(double t, double a, double b) { return a + t * (b - a); }
__device__ __forceinline__ double mc_clamped_lerp(double a, double b, double t) {
    if (t < 0.0) return a;
    if (t > 1.0) return b;
    return mc_lerp(t, a, b);
}
__device__ __forceinline__ double mc_lerp_progress(double v, double a, double b) { return (v - a) / (b - a); }
__device__ __forceinline__ double mc_lerp_from_progress(double v, double mn, double mx, double a, double b) {
    return mc_lerp(mc_lerp_progress(v, mn, mx), a, b);
}
__device__ __forceinline__ int floor_div(int a, int b) {
    int q = a / b, r = a % b;
    if (r != 0 && ((r < 0) != (b < 0))) q--;
    return q;
}
__device__ __forceinline__ double ygrad(double y, double from_y, double to_y, double from_v, double to_v) {
    double t = mc_clamp((y - from_y) / (to_y - from_y), 0.0, 1.0);
    return mc_lerp(t, from_v, to_v);
}

// x^3 rounded once (the reference calls pow(x, 3.0), which glibc rounds correctly): the exact
// square as a double-double (Dekker's two-product, with the fused multiply-add used only to
// recover the rounding error exactly), then the exact cube's leading parts summed once.
__device__ __forceinline__ double cube_rn(double x) {
    double s = x * x;
    double se = __fma_rn(x, x, -s);          // x*x = s + se exactly
    double c1 = s * x;
    double c1e = __fma_rn(s, x, -c1);        // s*x = c1 + c1e exactly
    double c2 = se * x;                      // tail of the cube (its own rounding is far below 1 ulp of c1)
    return c1 + (c1e + c2);
}

// ------------------------------------------------------------------------------------
// Perlin sampling (noise.c:200-290)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double gsel(uint32_t codes, int h) {
    const uint32_t c = (codes >> (2 * h)) & 3u;
    return c == 1u ? 1.0 : (c == 3u ? -1.0 : 0.0);
}
__device__ __forceinline__ double p2_grad(int hash, double x, double y, double z) {
    const int h = hash & 15;
    return gsel(kGradCodeX, h) * x + gsel(kGradCodeY, h) * y + gsel(kGradCodeZ, h) * z;
}

__device__ double p2_perlin_at(const P2Perlin &P, int i, int j, int k, double x, double y, double z,
                               double fade_y_of) {
    const uint8_t *pm = P.perm;
    int a = pm[i & 255], b = pm[(i + 1) & 255];
    int c = pm[(a + j) & 255], d = pm[(a + j + 1) & 255];
    int e = pm[(b + j) & 255], f = pm[(b + j + 1) & 255];
    double v000 = p2_grad(pm[(c + k) & 255], x, y, z);
    double v100 = p2_grad(pm[(e + k) & 255], x - 1, y, z);
    double v010 = p2_grad(pm[(d + k) & 255], x, y - 1, z);
    double v110 = p2_grad(pm[(f + k) & 255], x - 1, y - 1, z);
    double v001 = p2_grad(pm[(c + k + 1) & 255], x, y, z - 1);
    double v101 = p2_grad(pm[(e + k + 1) & 255], x - 1, y, z - 1);
    double v011 = p2_grad(pm[(d + k + 1) & 255], x, y - 1, z - 1);
    double v111 = p2_grad(pm[(f + k + 1) & 255], x - 1, y - 1, z - 1);
    double fx = fade(x), fy = fade(fade_y_of), fz = fade(z);
    double x00 = lerp(fx, v000, v100), x10 = lerp(fx, v010, v110);
    double x01 = lerp(fx, v001, v101), x11 = lerp(fx, v011, v111);
    return lerp(fz, lerp(fy, x00, x10), lerp(fy, x01, x11));
}

// lysh_perlin_sample (noise.c:234-250): y_scale / y_max fold the y coordinate (legacy octaves).
__device__ double p2_perlin(const P2Perlin &P, double x, double y, double z, double ys, double ymax) {
    double d = x + P.ox, e = y + P.oy, f = z + P.oz;
    int i = (int)floor(d), j = (int)floor(e), k = (int)floor(f);
    double g = d - i, h = e - j, l = f - k;
    double m;
    if (ys != 0.0) {
        double nn = (ymax >= 0.0 && ymax < h) ? ymax : h;
        m = floor(nn / ys + 1.0000000116860974E-7) * ys;
    } else {
        m = 0.0;
    }
    return p2_perlin_at(P, i, j, k, g, h - m, l, h);
}

__device__ double p2_octaves(const P2World &W, const P2Spec &S, int sub, double x, double y, double z) {
    double value = 0.0;
    const P2Perlin *base = W.perl + S.first_slot + sub * S.npresent;
    for (int p = 0; p < S.npresent; p++) {
        const double lac = S.lac[p];
        double v = p2_perlin(base[p], keep_precision(x * lac), keep_precision(y * lac), keep_precision(z * lac),
                             0.0, 0.0);
        value += (S.amp[p] * v) * S.per[p];
    }
    return value;
}

__device__ double p2_dbl(const P2Tables &T, const P2World &W, int q, double x, double y, double z) {
    const P2Spec &S = T.spec[W.large][q];
    return (p2_octaves(W, S, 0, x, y, z) + p2_octaves(W, S, 1, x * kDblScale, y * kDblScale, z * kDblScale)) *
           S.amplitude;
}

// ------------------------------------------------------------------------------------
// Splines and terrain (spline.c, terrain.c)
// ------------------------------------------------------------------------------------
__device__ int spline_lower_bound(const float *loc, int n, float v) {
    int start = 0, len = n;
    while (len > 0) {
        int half = len / 2;
        int mid = start + half;
        if (v < loc[mid]) {
            len = half;
        } else {
            start = mid + 1;
            len -= half + 1;
        }
    }
    return start;
}
__device__ __forceinline__ float lerpf(float t, float a, float b) { return a + t * (b - a); }

// CubicSpline.apply over the nested spline table (spline.c:26-57), evaluated with an explicit
// stack instead of recursion: each frame is one node waiting for its first and second child.
// The host checks at upload that the table nests no deeper than kSplineDepth.
__device__ float p2_spline(const P2Tables &T, int root, const float *pt) {
    int node[kSplineDepth], stage[kSplineDepth];
    float first[kSplineDepth];
    int sp = 0;
    node[0] = root;
    stage[0] = 0;
    float ret = 0.0f;
    for (;;) {
        const SplineNode &n = T.nodes[node[sp]];
        float result;
        if (n.kind == 1) {
            result = n.constant;
        } else {
            const float f = pt[n.coord];
            const float *loc = T.floats + n.loc;
            const float *der = T.floats + n.der;
            const int *ch = T.child + n.child;
            const int i = spline_lower_bound(loc, n.n, f) - 1;
            const int j = n.n - 1;
            if (i < 0 || i == j) {   // outside the points: the end child plus a linear extension
                const int k = i < 0 ? 0 : j;
                if (stage[sp] == 0) {
                    if (sp + 1 >= kSplineDepth) return __int_as_float(0x7FC00000);
                    stage[sp] = 1;
                    node[sp + 1] = ch[k];
                    stage[sp + 1] = 0;
                    sp++;
                    continue;
                }
                result = ret + der[k] * (f - loc[k]);
            } else {
                if (stage[sp] < 2) {
                    if (sp + 1 >= kSplineDepth) return __int_as_float(0x7FC00000);
                    if (stage[sp] == 1) first[sp] = ret;
                    node[sp + 1] = ch[i + stage[sp]];
                    stage[sp]++;
                    stage[sp + 1] = 0;
                    sp++;
                    continue;
                }
                const float g = loc[i], h = loc[i + 1];
                const float k = (f - g) / (h - g);
                const float l = first[sp], m = ret;
                const float d1 = der[i], d2 = der[i + 1];
                const float pp = d1 * (h - g) - (m - l);
                const float qq = -d2 * (h - g) + (m - l);
                result = lerpf(k, l, m) + k * (1.0f - k) * lerpf(k, pp, qq);
            }
        }
        if (sp == 0) return result;
        ret = result;
        sp--;
    }
}

__device__ __forceinline__ float normalized_weirdness_118(float w) {
    float a = w < 0.0f ? -w : w;
    float b = a - 0.6666667f;
    float c = b < 0.0f ? -b : b;
    float d = c - 0.33333334f;
    return -d * 3.0f;
}
__device__ __forceinline__ float normalized_weirdness_261(double w) {
    double a = fabs(w);
    double b = -0.6666666666666666 + a;
    double c = fabs(b);
    double d = -0.3333333333333333 + c;
    return (float)(-3.0 * d);
}

struct TerrainInfo {
    double sx, sz;          // shifted coordinates
    double c, w, e;         // continentalness, weirdness, erosion
};

__device__ void p2_terrain(const P2Tables &T, const P2World &W, int bx, int bz, TerrainInfo &ti) {
    ti.sx = (double)bx + p2_dbl(T, W, Q_OFFSET, (double)bx, 0.0, (double)bz) * 4.0;
    ti.sz = (double)bz + p2_dbl(T, W, Q_OFFSET, (double)bz, (double)bx, 0.0) * 4.0;
    ti.c = p2_dbl(T, W, Q_CONT, ti.sx, 0.0, ti.sz);
    ti.w = p2_dbl(T, W, Q_RIDGE, ti.sx, 0.0, ti.sz);
    ti.e = p2_dbl(T, W, Q_EROSION, ti.sx, 0.0, ti.sz);
}

// TerrainNoisePoint with the 26.1 ridges_folded (spline.c:112-126).
struct TerrainPoint {
    float offset, factor, peaks;
};
__device__ TerrainPoint p2_point_261(const P2Tables &T, const TerrainInfo &ti) {
    float pt[4] = {(float)ti.c, (float)ti.e, normalized_weirdness_261(ti.w), (float)ti.w};
    TerrainPoint p;
    p.offset = p2_spline(T, T.root_offset, pt) + (-0.50375f);
    p.factor = p2_spline(T, T.root_factor, pt);
    p.peaks = p2_spline(T, T.root_peak, pt);
    return p;
}

// column_top.c ps_offset_factor: the density-function offset / factor in double.
__device__ void p2_offset_factor(const P2Tables &T, const TerrainInfo &ti, double &offset, double &factor) {
    const float w = (float)ti.w;
    float pt[4] = {(float)ti.c, (float)ti.e, normalized_weirdness_118(w), w};
    const double raw_offset = (double)p2_spline(T, T.root_offset, pt);
    const double raw_factor = (double)p2_spline(T, T.root_factor, pt);
    const double blend_alpha = 1.0, blend_offset = 0.0;
    offset = blend_offset * (1.0 + -1.0 * blend_alpha) + (-0.5037500262260437 + raw_offset) * blend_alpha;
    factor = 10.0 + blend_alpha * (-10.0 + raw_factor);
}

__device__ __forceinline__ double ps_density(double y, double offset, double factor) {
    double depth = ygrad(y, -64.0, 320.0, 1.5, -1.5) + offset;
    double v = depth * factor;
    double cheese = 4.0 * (v > 0.0 ? v : v * 0.25);
    double c = mc_clamp(-0.703125 + cheese, -64.0, 64.0);
    double a1 = ygrad(y, 240.0, 256.0, 1.0, 0.0);
    double a2 = ygrad(y, -64.0, -40.0, 0.0, 1.0);
    return -0.390625 + (0.1171875 + a2 * (-0.1171875 + (-0.078125 + a1 * (0.078125 + c))));
}

// lysh_preliminary_surface_level (column_top.c:94-118), block coordinates.
__device__ int p2_column_top(const P2Tables &T, const P2World &W, int x, int z) {
    TerrainInfo ti;
    p2_terrain(T, W, x >> 2, z >> 2, ti);
    double offset, factor;
    p2_offset_factor(T, ti, offset, factor);
    double inv = 1.0 / factor;
    double inner = inv * 0.2734375 + offset * -1.0;
    double ub = mc_clamp(128.0 + -128.0 * inner, -40.0, 320.0);
    int y = (int)(ub / 8.0) * 8;
    if (y <= -64) return -64;
    for (int i = y; i >= -64; i -= 8)
        if (ps_density((double)i, offset, factor) > 0.0) return i;
    return -64;
}

// ------------------------------------------------------------------------------------
// Blended base noise (interp_noise.c:100-139)
// ------------------------------------------------------------------------------------
__device__ double p2_blended(const P2Tables &T, const P2World &W, int x, int y, int z) {
    const P2Perlin *lower = W.perl + T.n_slots, *upper = lower + 16, *mainn = lower + 32;
    const double xz_mult = 684.412 * 0.25, y_mult = 684.412 * 0.125;
    const double xz_factor = 80.0, y_factor = 160.0, smear = 8.0;
    double d = (double)x * xz_mult;
    double e = (double)y * y_mult;
    double f = (double)z * xz_mult;
    double g = d / xz_factor;
    double h = e / y_factor;
    double i = f / xz_factor;
    double j = y_mult * smear;
    double k = j / y_factor;
    double n = 0.0, q = 1.0;
    for (int o = 0; o < 8; o++) {
        n += p2_perlin(mainn[o], keep_precision(g * q), keep_precision(h * q), keep_precision(i * q), k * q, h * q) / q;
        q /= 2.0;
    }
    double t = (n / 10.0 + 1.0) / 2.0;
    const bool skip_min = (t >= 1.0), skip_max = (t <= 0.0);
    double l = 0.0, m = 0.0;
    q = 1.0;
    for (int o = 0; o < 16; o++) {
        double xx = keep_precision(d * q), yy = keep_precision(e * q), zz = keep_precision(f * q);
        double ys = j * q, ymax = e * q;
        if (!skip_min) l += p2_perlin(lower[o], xx, yy, zz, ys, ymax) / q;
        if (!skip_max) m += p2_perlin(upper[o], xx, yy, zz, ys, ymax) / q;
        q /= 2.0;
    }
    return mc_clamped_lerp(l / 512.0, m / 512.0, t) / 128.0;
}

// ------------------------------------------------------------------------------------
// Density column (density.c)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double lfp(const P2Tables &T, const P2World &W, int q, double x, double y, double z,
                                      double a, double b) {
    return mc_lerp_from_progress(p2_dbl(T, W, q, x, y, z), -1.0, 1.0, a, b);
}
__device__ __forceinline__ double scale_tunnels(double v) {
    if (v < -0.5) return 0.75;
    if (v < 0.0) return 1.0;
    if (v < 0.5) return 1.5;
    return 2.0;
}
__device__ __forceinline__ double scale_caves(double v) {
    if (v < -0.75) return 0.5;
    if (v < -0.5) return 0.75;
    if (v < 0.5) return 1.0;
    if (v < 0.75) return 2.0;
    return 3.0;
}

__device__ double p2_jagged(const P2Tables &T, const P2World &W, double peaks, int x, int z) {
    if (peaks == 0.0) return 0.0;
    double n = p2_dbl(T, W, Q_JAGGED, (double)x * 1500.0, 0.0, (double)z * 1500.0);
    return n > 0.0 ? peaks * n : (peaks / 2.0) * n;
}

// lysh_sample_noise_column (density.c:226-281) with useJagged = 1, noNoiseCaves = 0; `jagged`
// is the column's precomputed lysh_jagged value.
__device__ double p2_noise_column(const P2Tables &T, const P2World &W, int x, int y, int z, const TerrainPoint &tp,
                                  double jagged, double base_noise) {
    const double X = (double)x, Y = (double)y, Z = (double)z;
    double depth = (1.0 - Y / 128.0) + (double)tp.offset;
    double dens = (depth + jagged) * (double)tp.factor;
    dens = dens > 0.0 ? dens * 4.0 : dens;
    double g = dens + base_noise;
    double cheese, spaghetti, pillar;
    if (g < -64.0) {
        cheese = g;
        spaghetti = 64.0;
        pillar = -64.0;
    } else {
        double i = g - 1.5625;
        const bool shallow = i < 0.0;
        // cave entrance
        double ce = p2_dbl(T, W, Q_ENTRANCE, X * 0.75, Y * 0.5, Z * 0.75);
        double cave_entrance = ce + 0.37 + mc_clamped_lerp(0.3, 0.0, (10.0 + Y) / 40.0);
        // spaghetti roughness
        double rm = lfp(T, W, Q_ROUGH_MOD, X, Y, Z, 0.0, 0.1);
        double rr = fabs(p2_dbl(T, W, Q_ROUGH, X, Y, Z));
        double rough = (0.4 - rr) * rm;
        // spaghetti 3d
        double rarity = p2_dbl(T, W, Q_SP3D_RARITY, (double)(x * 2), Y, (double)(z * 2));
        double e = scale_tunnels(rarity);
        double h = lfp(T, W, Q_SP3D_THICK, X, Y, Z, 0.065, 0.088);
        double l3 = p2_dbl(T, W, Q_SP3D_1, X / e, Y / e, Z / e);
        double m3 = fabs(e * l3) - h;
        double n3 = p2_dbl(T, W, Q_SP3D_2, X / e, Y / e, Z / e);
        double o3 = fabs(e * n3) - h;
        double sp3d = mc_clamp(jmax(m3, o3), -1.0, 1.0);
        double m = jmin(cave_entrance, sp3d + rough);
        if (shallow) {
            cheese = g;
            spaghetti = m * 5.0;
            pillar = -64.0;
        } else {
            double lv = p2_dbl(T, W, Q_LAYER, X, (double)(y * 8), Z);
            double layer = lv * lv * 4.0;
            if (layer > 64.0) {
                cheese = 64.0;
            } else {
                double raw = p2_dbl(T, W, Q_CHEESE, X, Y / 1.5, Z);
                double p = mc_clamp(raw + 0.27, -1.0, 1.0);
                double qv = i * 1.28;
                cheese = p + mc_clamped_lerp(0.5, 0.0, qv) + layer;
            }
            // spaghetti 2d
            double mod = p2_dbl(T, W, Q_SP2D_MOD, (double)(x * 2), Y, (double)(z * 2));
            double s = scale_caves(mod);
            double h2 = lfp(T, W, Q_SP2D_THICK, (double)(x * 2), Y, (double)(z * 2), 0.6, 1.3);
            double v2 = p2_dbl(T, W, Q_SP2D, X / s, Y / s, Z / s);
            double j2 = fabs(s * v2) - 0.083 * h2;
            double l2 = lfp(T, W, Q_SP2D_ELEV, X, 0.0, Z, (double)-8, 8.0);
            double m2 = fabs(l2 - Y / 8.0) - h2;
            m2 = m2 * m2 * m2;
            double sp2d = mc_clamp(jmax(m2, j2), -1.0, 1.0);
            spaghetti = jmin(m, sp2d + rough);
            // pillar
            double rare = lfp(T, W, Q_PILLAR_RARE, X, Y, Z, 0.0, 2.0);
            double thick = lfp(T, W, Q_PILLAR_THICK, X, Y, Z, 0.0, 1.1);
            thick = cube_rn(thick);
            double pf = p2_dbl(T, W, Q_PILLAR, X * 25.0, Y * 0.3, Z * 25.0);
            double pg = thick * (pf * 2.0 - rare);
            pillar = pg > 0.03 ? pg : -__longlong_as_double(0x7FF0000000000000LL);
        }
    }
    double v = jmax(jmin(cheese, spaghetti), pillar);
    // applySlides(v, y / 8) with C's truncating division
    const int cell_y = y / 8;
    const int iy = cell_y - (-8);
    {
        double dd = (double)((48 - iy) - 8) / (double)2;
        v = mc_clamped_lerp(-0.078125, v, dd);
    }
    {
        double dd = (double)(iy - 0) / (double)3;
        v = mc_clamped_lerp(0.1171875, v, dd);
    }
    return mc_clamp(v, -64.0, 64.0);
}

__device__ __forceinline__ double squeeze(double v) {
    double a = mc_clamp(v * 0.64, -1.0, 1.0);
    return a / 2.0 - a * a * a / 24.0;
}

__device__ __forceinline__ bool noodle_y_in_range(int y) { return y >= -60 && y <= 320; }

// lysh_noodle_child (density.c:185-205): which 0 = noodle, 1 = thickness, 2 = ridge a, 3 = ridge b.
__device__ double p2_noodle_child(const P2Tables &T, const P2World &W, int which, int x, int y, int z) {
    const double X = (double)x, Y = (double)y, Z = (double)z;
    switch (which) {
        case 0:
            if (!noodle_y_in_range(y)) return -1.0;
            return p2_dbl(T, W, Q_NOODLE, X, Y, Z);
        case 1:
            if (!noodle_y_in_range(y)) return 0.0;
            return -0.07500000000000001 + -0.025 * p2_dbl(T, W, Q_NOODLE_THICK, X, Y, Z);
        default:
            if (!noodle_y_in_range(y)) return 0.0;
            return p2_dbl(T, W, which == 2 ? Q_NOODLE_RA : Q_NOODLE_RB, X * 2.6666666666666665,
                          Y * 2.6666666666666665, Z * 2.6666666666666665);
    }
}
__device__ __forceinline__ double noodle_combine(double n, double thickness, double ra, double rb) {
    if (n >= -1000000.0 && n < 0.0) return 64.0;
    return thickness + 1.5 * jmax(fabs(ra), fabs(rb));
}

// lysh_phase2_density_raw_at (phase2.c:151-158)
__device__ double p2_density_raw(const P2Tables &T, const P2World &W, int x, int y, int z) {
    TerrainInfo ti;
    p2_terrain(T, W, x >> 2, z >> 2, ti);
    TerrainPoint tp = p2_point_261(T, ti);
    double base = p2_blended(T, W, x, y, z);
    double jag = p2_jagged(T, W, (double)tp.peaks, x, z);
    return p2_noise_column(T, W, x, y, z, tp, jag, base);
}

// ------------------------------------------------------------------------------------
// Interpolated density over the chunk grid (phase2.c:44-194)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double interp_grid(const double (*grid)[kGridYs], int cell_x, int cell_z, int rel_x,
                                              int rel_y, int rel_z, int cy) {
    const int gx = cell_x & 3, gz = cell_z & 3;
    const double *c00 = grid[gx * 5 + gz];
    const double *c10 = grid[(gx + 1) * 5 + gz];
    const double *c01 = grid[gx * 5 + gz + 1];
    const double *c11 = grid[(gx + 1) * 5 + gz + 1];
    const double dx = (double)rel_x / 4.0, dy = (double)rel_y / 8.0, dz = (double)rel_z / 4.0;
    double xz00 = mc_lerp(dy, c00[cy], c00[cy + 1]);
    double xz10 = mc_lerp(dy, c10[cy], c10[cy + 1]);
    double xz01 = mc_lerp(dy, c01[cy], c01[cy + 1]);
    double xz11 = mc_lerp(dy, c11[cy], c11[cy + 1]);
    double z0 = mc_lerp(dx, xz00, xz10);
    double z1 = mc_lerp(dx, xz01, xz11);
    return mc_lerp(dz, z0, z1);
}

// lysh_phase2_density_at for a block of the job's chunk.
__device__ double p2_density_at(const P2Tables &T, const P2World &W, const P2Chunk &J, int x, int y, int z) {
    const int y_off = y + 64;
    if (y_off < 0 || y_off >= 384) return p2_density_raw(T, W, x, y, z);
    const int cell_x = x >> 2, cell_z = z >> 2, rel_x = x & 3, rel_z = z & 3;
    const int cy = y_off / 8, rel_y = y_off - cy * 8;
    double v = interp_grid(J.main, cell_x, cell_z, rel_x, rel_y, rel_z, cy);
    double sq = squeeze(v);
    double nn = p2_noodle_child(T, W, 0, x, y, z);
    double th = interp_grid(J.noodle[0], cell_x, cell_z, rel_x, rel_y, rel_z, cy);
    double ra = interp_grid(J.noodle[1], cell_x, cell_z, rel_x, rel_y, rel_z, cy);
    double rb = interp_grid(J.noodle[2], cell_x, cell_z, rel_x, rel_y, rel_z, cy);
    return jmin(sq, noodle_combine(nn, th, ra, rb));
}

// ------------------------------------------------------------------------------------
// Aquifer (aquifer.c, 26.1 NoiseBasedAquifer)
// ------------------------------------------------------------------------------------
constexpr int kNoFluidY = -32512;

__device__ __forceinline__ void global_fluid(int y, int &level, int &type) {
    if (y < -54) {
        level = -54;
        type = BS_LAVA;
    } else {
        level = 63;
        type = BS_WATER;
    }
}
__device__ __forceinline__ int level_block_at(int level, int type, int y) { return y < level ? type : BS_AIR; }

__device__ bool deep_dark(const P2Tables &T, const P2World &W, int x, int y, int z) {
    TerrainInfo ti;
    p2_terrain(T, W, x >> 2, z >> 2, ti);
    if (!(ti.e < -0.22499999403953552)) return false;
    double offset, factor;
    p2_offset_factor(T, ti, offset, factor);
    double depth = ygrad((double)y, -64.0, 320.0, 1.5, -1.5) + offset;
    return depth > 0.8999999761581421;
}

__device__ const int kSurfOffsets[13][2] = {{0, 0},   {-2, -1}, {-1, -1}, {0, -1}, {1, -1}, {-3, 0}, {-2, 0},
                                           {-1, 0}, {1, 0},    {-2, 1},  {-1, 1}, {0, 1},  {1, 1}};

// The column top of block column (x, z): from the chunk's table (J non-null) where the column lies
// in it, else computed.
__device__ __forceinline__ int p2_top(const P2Tables &T, const P2World &W, const P2Chunk *J, int x, int z) {
    if (J) {
        const int qx = (x >> 2) - (4 * J->chunk_x - 16), qz = (z >> 2) - (4 * J->chunk_z - 8);
        if ((unsigned)qx < (unsigned)kTopX && (unsigned)qz < (unsigned)kTopZ) return J->tops[qz][qx];
    }
    return p2_column_top(T, W, x, z);
}

// computeFluid (aquifer.c:327-376): level and type; the column tops come from the job's table when
// J is given.
__device__ void p2_compute_fluid(const P2Tables &T, const P2World &W, const P2Chunk *J, int x, int y, int z,
                                 int &out_level, int &out_type) {
    int glevel, gtype;
    global_fluid(y, glevel, gtype);
    int min_top = 0x7FFFFFFF;
    bool has_above = false;
    for (int i = 0; i < 13; i++) {
        const int bx = x + kSurfOffsets[i][0] * 16, bz = z + kSurfOffsets[i][1] * 16;
        const int top = p2_top(T, W, J, bx, bz);
        const int top_adj = top + 8;
        const bool center = (i == 0);
        if (center && y - 12 > top_adj) {
            out_level = glevel;
            out_type = gtype;
            return;
        }
        const bool above = y + 12 > top_adj;
        if (above || center) {
            int lvl, typ;
            global_fluid(top_adj, lvl, typ);
            if (level_block_at(lvl, typ, top_adj) != BS_AIR) {
                if (center) has_above = true;
                if (above) {
                    out_level = lvl;
                    out_type = typ;
                    return;
                }
            }
        }
        if (top < min_top) min_top = top;
    }
    // computeSurfaceLevel
    int level;
    if (deep_dark(T, W, x, y, z)) {
        level = kNoFluidY;
    } else {
        const int d = (min_top + 8) - y;
        const double f = has_above ? mc_clamped_lerp(1.0, 0.0, mc_lerp_progress((double)d, 0.0, 64.0)) : 0.0;
        const double high = mc_lerp_from_progress(f, 1.0, 0.0, -0.3, 0.8);
        const double low = mc_lerp_from_progress(f, 1.0, 0.0, -0.8, 0.4);
        const double flood = mc_clamp(p2_dbl(T, W, Q_AQ_FLOOD, (double)x, (double)y * 0.67, (double)z), -1.0, 1.0);
        if (flood - high > 0.0) {
            level = glevel;
        } else if (flood - low > 0.0) {
            const int fx = floor_div(x, 16), fy = floor_div(y, 40), fz = floor_div(z, 16);
            const int base = fy * 40 + 20;
            const double n = p2_dbl(T, W, Q_AQ_SPREAD, (double)fx, (double)fy * 0.7142857142857143, (double)fz) * 10.0;
            const int q = (int)floor(n / 3.0) * 3;
            const int lv = base + q;
            level = min_top < lv ? min_top : lv;
        } else {
            level = kNoFluidY;
        }
    }
    // computeFluidType
    int type = gtype;
    if (level <= -10 && level != kNoFluidY && gtype != BS_LAVA) {
        const int bx = floor_div(x, 64), by = floor_div(y, 40), bz = floor_div(z, 64);
        const double n = p2_dbl(T, W, Q_AQ_LAVA, (double)bx, (double)by, (double)bz);
        if (fabs(n) > 0.3) type = BS_LAVA;
    }
    out_level = level;
    out_type = type;
}

__device__ __forceinline__ int64_t mc_hash_code(int x, int y, int z) {
    const int64_t xm = (int64_t)(int32_t)((uint32_t)x * 3129871u);
    uint64_t i = (uint64_t)(xm ^ ((int64_t)z * 116129781LL) ^ (int64_t)y);
    i = i * i * 42317861ULL + i * 11ULL;
    return (int64_t)i >> 16;
}

__device__ __forceinline__ int aq_index(const P2Chunk &J, int gx, int gy, int gz) {
    const int dx = gx - J.min_gx, dy = gy - J.min_gy, dz = gz - J.min_gz;
    if (dx < 0 || dx >= kAqX || dy < 0 || dy >= kAqY || dz < 0 || dz >= kAqZ) return -1;
    return (dy * kAqZ + dz) * kAqX + dx;
}

__device__ __forceinline__ double similarity(int a, int b) { return 1.0 - (double)(b - a) / 25.0; }

__device__ double aq_pressure(const P2Tables &T, const P2World &W, int x, int y, int z, bool &have, double &acc,
                              int la, int ta, int lb, int tb) {
    const int sa = level_block_at(la, ta, y), sb = level_block_at(lb, tb, y);
    if ((sa == BS_LAVA && sb == BS_WATER) || (sa == BS_WATER && sb == BS_LAVA)) return 2.0;
    int dy = la - lb;
    if (dy < 0) dy = -dy;
    if (dy == 0) return 0.0;
    const double mid = 0.5 * ((double)la + (double)lb);
    const double f = ((double)y + 0.5) - mid;
    const double half = (double)dy / 2.0;
    const double n = half - fabs(f);
    double o;
    if (f > 0.0) {
        const double p = 0.0 + n;
        o = p > 0.0 ? p / 1.5 : p / 2.5;
    } else {
        const double p = 3.0 + n;
        o = p > 0.0 ? p / 3.0 : p / 10.0;
    }
    double inner;
    if (o < -2.0 || o > 2.0) {
        inner = 0.0;
    } else if (!have) {
        acc = p2_dbl(T, W, Q_AQ_BARRIER, (double)x, (double)y * 0.5, (double)z);
        have = true;
        inner = acc;
    } else {
        inner = acc;
    }
    return 2.0 * (inner + o);
}

// Aquifer.computeSubstance (aquifer.c:438-563) on the job's precomputed cells; BS_SOLID = null.
__device__ int p2_substance(const P2Tables &T, const P2World &W, const P2Chunk &J, int x, int y, int z,
                            double density) {
    if (density > 0.0) return BS_SOLID;
    int glevel, gtype;
    global_fluid(y, glevel, gtype);
    // skipSamplingAboveY from the highest column top around the chunk
    const int skip_above = (floor_div((J.max_psl + 8) + 12, 12) + 1) * 12 + 11 - 1;
    if (y > skip_above) return level_block_at(glevel, gtype, y);
    if (level_block_at(glevel, gtype, y) == BS_LAVA) return BS_LAVA;
    const int gx = floor_div(x - 5, 16), gy = floor_div(y + 1, 12), gz = floor_div(z - 5, 16);
    int d[4] = {0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF};
    int slot[4] = {0, 0, 0, 0};
    for (int i = 0; i <= 1; i++)
        for (int j = -1; j <= 1; j++)
            for (int k = 0; k <= 1; k++) {
                const int idx = aq_index(J, gx + i, gy + j, gz + k);
                if (idx < 0) continue;
                const int64_t pk = J.aq_loc[idx];
                const int px = (int)(pk >> 38), py = (int)((pk << 52) >> 52), pz = (int)((pk << 26) >> 38);
                const int dx = px - x, dy = py - y, dz = pz - z;
                const int dist = dx * dx + dy * dy + dz * dz;
                if (dist <= d[0]) {
                    d[3] = d[2]; d[2] = d[1]; d[1] = d[0]; d[0] = dist;
                    slot[3] = slot[2]; slot[2] = slot[1]; slot[1] = slot[0]; slot[0] = idx;
                } else if (dist <= d[1]) {
                    d[3] = d[2]; d[2] = d[1]; d[1] = dist;
                    slot[3] = slot[2]; slot[2] = slot[1]; slot[1] = idx;
                } else if (dist <= d[2]) {
                    d[3] = d[2]; d[2] = dist;
                    slot[3] = slot[2]; slot[2] = idx;
                } else if (dist <= d[3]) {
                    d[3] = dist;
                    slot[3] = idx;
                }
            }
    const int l0 = J.aq_level[slot[0]], t0 = J.aq_type[slot[0]];
    const double s01 = similarity(d[0], d[1]);
    const int result = level_block_at(l0, t0, y);
    if (!(s01 > 0.0)) return result;
    {
        int bl, bt;
        global_fluid(y - 1, bl, bt);
        if (result == BS_WATER && level_block_at(bl, bt, y - 1) == BS_LAVA) return result;
    }
    bool have = false;
    double acc = 0.0;
    const int l1 = J.aq_level[slot[1]], t1 = J.aq_type[slot[1]];
    const double p1 = s01 * aq_pressure(T, W, x, y, z, have, acc, l0, t0, l1, t1);
    if (density + p1 > 0.0) return BS_SOLID;
    const int l2 = J.aq_level[slot[2]], t2 = J.aq_type[slot[2]];
    const double s02 = similarity(d[0], d[2]);
    if (s02 > 0.0) {
        const double p2 = s01 * s02 * aq_pressure(T, W, x, y, z, have, acc, l0, t0, l2, t2);
        if (density + p2 > 0.0) return BS_SOLID;
    }
    const double s12 = similarity(d[1], d[2]);
    if (s12 > 0.0) {
        const double p3 = s01 * s12 * aq_pressure(T, W, x, y, z, have, acc, l1, t1, l2, t2);
        if (density + p3 > 0.0) return BS_SOLID;
    }
    return result;
}

// lysh_phase2_block_at: the pre-carver block state.
__device__ __forceinline__ int p2_block_at(const P2Tables &T, const P2World &W, const P2Chunk &J, int x, int y,
                                           int z) {
    return p2_substance(T, W, J, x, y, z, p2_density_at(T, W, J, x, y, z));
}

__device__ __forceinline__ int carve_index(int lx, int y, int lz) { return ((lz & 15) << 4) | (lx & 15) | ((y + 64) << 8); }

// Surface height (NOT_AIR predicate, y + 1; phase2.c:318-334 and :438-456) of a column of the job's
// chunk, from the job's per-block states (p2_states_kernel).  The 384 levels are read sixteen at a
// time (independent loads) and tested top-down in order.
__device__ int p2_height(const P2Tables &T, const P2World &W, const P2Chunk &J, int x, int z, bool carved) {
    (void)T;
    (void)W;
    constexpr int kGroup = 16;
    static_assert((320 + 64) % kGroup == 0, "levels in whole groups");
    for (int y0 = 319; y0 >= -64; y0 -= kGroup) {
        uint8_t cv[kGroup], pre[kGroup];
#pragma unroll
        for (int k = 0; k < kGroup; k++) {
            const int ci = carve_index(x & 15, y0 - k, z & 15);
            cv[k] = carved ? J.cells[ci] : (uint8_t)CV_UNCHANGED;
            pre[k] = J.states[ci];
        }
#pragma unroll
        for (int k = 0; k < kGroup; k++) {
            const int st = cv[k] != CV_UNCHANGED ? (int)cv[k] : (int)(pre[k] & 15u);   // CV_* = BS_* codes
            if (st != BS_AIR) return y0 - k + 1;
        }
    }
    return -64;
}

// Every block of every job's chunk: its pre-carver state and its aquifer substance at density 0,
// the two things the carvers and the height scans read per block.  One thread per block: these
// are independent, where the carvers and the column scans are serial chains per chunk / column.
__global__ void __launch_bounds__(256) p2_states_kernel(const P2Tables *__restrict__ Tp,
                                                        const P2World *__restrict__ worlds, P2Chunk *jobs) {
    P2Chunk &J = jobs[blockIdx.y];
    const P2Tables &T = *Tp;
    const P2World &W = worlds[J.world];
    const int q = blockIdx.x * 256 + threadIdx.x;   // carve_index(lx, y, lz)
    const int x = J.chunk_x * 16 + (q & 15), z = J.chunk_z * 16 + ((q >> 4) & 15), y = (q >> 8) - 64;
    const int nat = p2_block_at(T, W, J, x, y, z);
    const int sub = y > -56 ? p2_substance(T, W, J, x, y, z, 0.0) : BS_LAVA;
    J.states[q] = (uint8_t)(nat | (sub << 4));
    J.cells[q] = (uint8_t)CV_UNCHANGED;   // the carvers' working copy starts untouched
}

// ------------------------------------------------------------------------------------
// Kernels: world construction
// ------------------------------------------------------------------------------------
__device__ void walk_perlin(Xr &r) {
    (void)xr_next(r);
    (void)xr_next(r);
    (void)xr_next(r);
    for (int i = 0; i < 256; i++) (void)xr_bounded(r, (uint32_t)(256 - i));
}

// Whether walk_perlin from r would take a second draw for any of its bounded draws.
__device__ bool walk_perlin_rejects(Xr r) {
    (void)xr_next(r);
    (void)xr_next(r);
    (void)xr_next(r);
    for (int i = 0; i < 256; i++) {
        const uint32_t bound = (uint32_t)(256 - i);
        const uint64_t v = (uint64_t)(uint32_t)xr_next(r) * bound;
        if ((uint32_t)v < bound && (uint32_t)v < (0u - bound) % bound) return true;
    }
    return false;
}

// One CTA per world: start states of the 40 legacy octaves (created in sequence from the
// "minecraft:terrain" random, lower -> upper -> main; interp_noise.c:44-75, noise.c:205-250)
// and the aquifer's positional random factory (aquifer.c:126-136).  An octave's walk takes 259
// draws unless a bounded draw rejects (odds below 1e-7 per draw), so thread k jumps the stream's
// state 259 k steps (a GF(2) matrix over the 128-bit state) and checks its own octave's draws;
// if any octave rejects, thread 0 walks the stream in order instead.
__global__ void __launch_bounds__(64) p2_legacy_kernel(const P2Tables *__restrict__ Tp, P2World *worlds) {
    __shared__ int rejected;
    const P2Tables &T = *Tp;
    P2World &W = worlds[blockIdx.x];
    const int k = threadIdx.x;
    if (k == 0) rejected = 0;
    __syncthreads();
    const Xr fork = seed_fork_of(W.seed);
    const Xr r0 = xr_make(T.terrain_lo ^ fork.lo, T.terrain_hi ^ fork.hi);
    if (k < kLegacyPerlins) {
        const ulonglong2 *J = reinterpret_cast<const ulonglong2 *>(T.legacy_jump) + (size_t)k * 128;
        Xr r{0, 0};
#pragma unroll 8
        for (int b = 0; b < 64; b++) {
            const ulonglong2 m = J[b];
            r.lo |= (uint64_t)(__popcll((m.x & r0.lo) ^ (m.y & r0.hi)) & 1) << b;
        }
#pragma unroll 8
        for (int b = 0; b < 64; b++) {
            const ulonglong2 m = J[64 + b];
            r.hi |= (uint64_t)(__popcll((m.x & r0.lo) ^ (m.y & r0.hi)) & 1) << b;
        }
        W.legacy_rng[k] = r;
        if (walk_perlin_rejects(r)) atomicOr(&rejected, 1);
    }
    __syncthreads();
    if (k != 0) return;
    if (rejected) {
        Xr r = r0;
        for (int q = 0; q < kLegacyPerlins; q++) {
            W.legacy_rng[q] = r;
            walk_perlin(r);
        }
    }
    Xr s = xr_from_seed(W.seed);
    Xr base;
    base.lo = xr_next(s);
    base.hi = xr_next(s);
    Xr aq = xr_make(T.aquifer_lo ^ base.lo, T.aquifer_hi ^ base.hi);
    W.aq_rand_lo = xr_next(aq);
    W.aq_rand_hi = xr_next(aq);
}

constexpr int kBuildThreads = 128;

// One thread per Perlin table of one world.
__global__ void __launch_bounds__(kBuildThreads) p2_build_kernel(const P2Tables *__restrict__ Tp, P2World *worlds) {
    __shared__ uint8_t col[256 * kBuildThreads];
    const P2Tables &T = *Tp;
    P2World &W = worlds[blockIdx.y];
    const int slot = blockIdx.x * kBuildThreads + threadIdx.x;
    const int n_total = T.n_slots + kLegacyPerlins;
    uint8_t *t = col + threadIdx.x;
    for (int k = 0; k < 256; k++) t[k * kBuildThreads] = (uint8_t)k;
    if (slot >= n_total) return;
    Xr r;
    if (slot < T.n_slots) {
        const int q = T.slot_noise[slot], sub = T.slot_sub[slot], p = T.slot_oct[slot];
        const P2Digest &D = T.digest[W.large][q];
        const Xr fork = seed_fork_of(W.seed);
        Xr noise = xr_make(D.name_lo ^ fork.lo, D.name_hi ^ fork.hi);
        uint64_t a = xr_next(noise), b = xr_next(noise);
        if (sub) {
            a = xr_next(noise);
            b = xr_next(noise);
        }
        const Xr sf = xr_make(a, b);
        r = xr_make(D.oct_lo[p] ^ sf.lo, D.oct_hi[p] ^ sf.hi);
    } else {
        r = W.legacy_rng[slot - T.n_slots];
    }
    P2Perlin &P = W.perl[slot];
    P.ox = xr_double(r) * 256.0;
    P.oy = xr_double(r) * 256.0;
    P.oz = xr_double(r) * 256.0;
    for (int i = 0; i < 256; i++) {
        const int j = i + xr_bounded(r, (uint32_t)(256 - i));
        const uint8_t a = t[i * kBuildThreads], b = t[j * kBuildThreads];
        t[i * kBuildThreads] = b;
        t[j * kBuildThreads] = a;
    }
    uint32_t *out = reinterpret_cast<uint32_t *>(P.perm);
    for (int k = 0; k < 64; k++)
        out[k] = (uint32_t)t[(4 * k) * kBuildThreads] | ((uint32_t)t[(4 * k + 1) * kBuildThreads] << 8) |
                 ((uint32_t)t[(4 * k + 2) * kBuildThreads] << 16) | ((uint32_t)t[(4 * k + 3) * kBuildThreads] << 24);
}

// ------------------------------------------------------------------------------------
// Kernels: chunk grid and aquifer cells
// ------------------------------------------------------------------------------------
constexpr int kGridThreads = 256;

// One CTA per job: the 25 corner columns' terrain points and jagged values, then 25 x 49 base
// densities and 3 x 25 x 49 noodle children (phase2.c:73-116).
__global__ void __launch_bounds__(kGridThreads) p2_grid_kernel(const P2Tables *__restrict__ Tp,
                                                               const P2World *__restrict__ worlds, P2Chunk *jobs) {
    // CTA (job, gx): the five corner columns c = gx * 5 + k of one cell row, so a job's grid is five
    // short chains on five SMs instead of one long one.  Threads 0..4 evaluate the columns' terrain
    // points while the others take the samples that do not need them (the blended noise of every
    // main sample and the three noodle children); the density columns follow the barrier.
    __shared__ TerrainPoint tp[5];
    __shared__ double jag[5];
    __shared__ double base[5 * kGridYs];
    const P2Tables &T = *Tp;
    P2Chunk &J = jobs[blockIdx.x];
    const P2World &W = worlds[J.world];
    const int gx = blockIdx.y;
    const int cx0 = J.chunk_x * 4, cz0 = J.chunk_z * 4;   // first cell of the chunk
    const int t = threadIdx.x;
    if (t < 5) {
        const int cell_x = cx0 + gx, cell_z = cz0 + t;
        TerrainInfo ti;
        p2_terrain(T, W, cell_x, cell_z, ti);
        tp[t] = p2_point_261(T, ti);
        jag[t] = p2_jagged(T, W, (double)tp[t].peaks, cell_x * 4, cell_z * 4);
    } else {
        for (int q = t - 5; q < 4 * 5 * kGridYs; q += (int)blockDim.x - 5) {
            const int which = q / (5 * kGridYs), rem = q % (5 * kGridYs);   // 0: main, 1..3: noodle
            const int k = rem / kGridYs, i = rem % kGridYs, c = gx * 5 + k;
            const int bx = (cx0 + gx) * 4, bz = (cz0 + k) * 4, y = -64 + i * 8;
            if (which == 0) base[rem] = p2_blended(T, W, bx, y, bz);
            else J.noodle[which - 1][c][i] = p2_noodle_child(T, W, which, bx, y, bz);
        }
    }
    __syncthreads();
    for (int q = t; q < 5 * kGridYs; q += blockDim.x) {
        const int k = q / kGridYs, i = q % kGridYs, c = gx * 5 + k;
        const int bx = (cx0 + gx) * 4, bz = (cz0 + k) * 4, y = -64 + i * 8;
        J.main[c][i] = p2_noise_column(T, W, bx, y, bz, tp[k], jag[k], base[q]);
    }
}

constexpr int kAqThreads = 128;

// Every column top of the job's table (one thread each) and their maximum over the grid's x/z
// span, from which skipSamplingAboveY derives (aquifer.c:158-196, column_top.c:94-118).
// CTA (job, part) of gridDim.y takes every gridDim.y-th entry.
__global__ void __launch_bounds__(kAqThreads) p2_tops_kernel(const P2Tables *__restrict__ Tp,
                                                             const P2World *__restrict__ worlds, P2Chunk *jobs) {
    const P2Tables &T = *Tp;
    P2Chunk &J = jobs[blockIdx.x];
    const P2World &W = worlds[J.world];
    const int part = blockIdx.y, parts = gridDim.y;
    const int min_bx = J.chunk_x * 16, min_bz = J.chunk_z * 16;
    const int min_gx = (min_bx - 5) >> 4, max_gx = ((min_bx + 15 - 5) >> 4) + 1;
    const int min_gz = (min_bz - 5) >> 4, max_gz = ((min_bz + 15 - 5) >> 4) + 1;
    if (part == 0 && threadIdx.x == 0) {
        J.min_gx = min_gx;
        J.min_gy = floor_div(-64 + 1, 12) - 1;
        J.min_gz = min_gz;
    }
    // skipSamplingAboveY's samples: x = x1 + 4 i <= x2, z = z1 + 4 j <= z2
    const int x1 = min_gx * 16, z1 = min_gz * 16, x2 = max_gx * 16 + 9, z2 = max_gz * 16 + 9;
    const int qx0 = 4 * J.chunk_x - 16, qz0 = 4 * J.chunk_z - 8;
    for (int q = part * (int)blockDim.x + (int)threadIdx.x; q < kTopX * kTopZ; q += parts * (int)blockDim.x) {
        const int x = (qx0 + q % kTopX) * 4, z = (qz0 + q / kTopX) * 4;
        const int top = p2_column_top(T, W, x, z);
        J.tops[q / kTopX][q % kTopX] = (int16_t)top;
        if (x >= x1 && x <= x2 && z >= z1 && z <= z2) atomicMax(&J.max_psl, top);
    }
}

// Every aquifer cell's random anchor and fluid status (aquifer.c:379-395, 481-501), computed up
// front; CTA (job, part) of gridDim.y takes every gridDim.y-th cell.
__global__ void __launch_bounds__(kAqThreads) p2_aquifer_kernel(const P2Tables *__restrict__ Tp,
                                                                const P2World *__restrict__ worlds, P2Chunk *jobs) {
    const P2Tables &T = *Tp;
    P2Chunk &J = jobs[blockIdx.x];
    const P2World &W = worlds[J.world];
    const int part = blockIdx.y, parts = gridDim.y;
    const int min_gx = J.min_gx, min_gy = J.min_gy, min_gz = J.min_gz;
    const Xr factory{W.aq_rand_lo, W.aq_rand_hi};
    for (int idx = part * (int)blockDim.x + (int)threadIdx.x; idx < kAqCells; idx += parts * (int)blockDim.x) {
        const int dx = idx % kAqX, dz = (idx / kAqX) % kAqZ, dy = idx / (kAqX * kAqZ);
        const int cx = min_gx + dx, cy = min_gy + dy, cz = min_gz + dz;
        Xr rnd = xr_make((uint64_t)mc_hash_code(cx, cy, cz) ^ factory.lo, factory.hi);
        const int px = (cx << 4) + xr_bounded(rnd, 10);
        const int py = cy * 12 + xr_bounded(rnd, 9);
        const int pz = (cz << 4) + xr_bounded(rnd, 10);
        const int64_t packed = ((int64_t)(px & 0x3FFFFFF) << 38) | ((int64_t)(pz & 0x3FFFFFF) << 12) |
                               (int64_t)(py & 0xFFF);
        J.aq_loc[idx] = packed;
        int level, type;
        p2_compute_fluid(T, W, &J, (int)(packed >> 38), (int)((packed << 52) >> 52), (int)((packed << 26) >> 38),
                         level, type);
        J.aq_level[idx] = level;
        J.aq_type[idx] = (uint8_t)type;
    }
}

// ------------------------------------------------------------------------------------
// Carvers (carver.c), one warp per job
// ------------------------------------------------------------------------------------
constexpr int kCarveThreads = 32;
constexpr int kMaskWords = kCarveCells / 32;

struct CarveCtx {
    const P2Tables *T;
    const P2World *W;
    const P2Chunk *J;
    uint8_t *cells;
    uint32_t *mask;
    float *width;                 // canyon width factors (384)
    double *fx, *fz, *fy;         // carve_ellipsoid's per-row / column / level offsets (shared)
    uint16_t *cols;               // its columns inside the ellipse (shared, 256)
    const float *sinq;            // Mth.SIN quarter wave (shared)
    float sin_half_turn;
    int tmin_x, tmin_z;
    double tmid_x, tmid_z;
};

// Mth.SIN[i] from the quarter wave in shared memory: entries 16385..32767 mirror 16383..1, the
// second half is the first negated, and entry 32768 is its own value.
// The walks copy the table's address into a SinTab by value, so that it stays in registers
// while the ellipsoid code stores through other pointers.
struct SinTab {
    const float *q;
    float half_turn;
};
__device__ __forceinline__ float sin_entry(const SinTab &t, int i) {
    const int h = i & 32767, k = h <= 16384 ? h : 32768 - h;
    float v = t.q[k];
    if (i & 32768) v = -v;
    return i == 32768 ? t.half_turn : v;
}
__device__ __forceinline__ float mc_sin(const SinTab &t, double a) {
    return sin_entry(t, (int)((long long)(a * 10430.378350470453) & 65535LL));
}
__device__ __forceinline__ float mc_cos(const SinTab &t, double a) {
    return sin_entry(t, (int)((long long)(a * 10430.378350470453 + 16384.0) & 65535LL));
}
__device__ __forceinline__ float lcg_float(uint64_t &st) { return (float)lcg_bits(st, 24) * 5.9604645e-8f; }
__device__ __forceinline__ float uniform_float(uint64_t &st, float lo, float hi) { return lcg_float(st) * (hi - lo) + lo; }
__device__ __forceinline__ void lcg_set_seed(uint64_t &st, uint64_t s) { st = (s ^ kLcgMul) & kLcgMask; }
__device__ __forceinline__ int jfloor(double d) { return (int)floor(d); }

// Skip-ahead for java.util.Random: k steps from state s give (A_k s + C_k) mod 2^48, so the
// fixed run of draws in one carver step comes from independent multiplies instead of a chain.
struct LcgJump {
    uint64_t a, c;
};
__host__ __device__ constexpr LcgJump lcg_jump(int k) {
    uint64_t a = 1, c = 0;
    for (int i = 0; i < k; i++) {
        a = (a * kLcgMul) & kLcgMask;
        c = (c * kLcgMul + 0xBULL) & kLcgMask;
    }
    return LcgJump{a, c};
}
template <int K>
__device__ __forceinline__ uint64_t lcg_ahead(uint64_t s) {
    constexpr LcgJump j = lcg_jump(K);
    return (s * j.a + j.c) & kLcgMask;
}
// nextFloat and nextInt(bound), bound a power of two, of the draw that produced state st
__device__ __forceinline__ float lcg_float_at(uint64_t st) {
    return (float)(int)(uint32_t)(st >> (48 - 24)) * 5.9604645e-8f;
}
__device__ __forceinline__ int lcg_int_pow2_at(uint64_t st, int bound) {
    return (int)(((int64_t)bound * (int64_t)(int)(uint32_t)(st >> (48 - 31))) >> 31);
}

// setLargeFeatureSeed (structure.c:26-42)
__device__ __forceinline__ uint64_t large_feature_state(uint64_t world_seed, int cx, int cz) {
    uint64_t st;
    lcg_set_seed(st, world_seed);
    const uint64_t a = lcg_long(st), b = lcg_long(st);
    const uint64_t s = (uint64_t)((int64_t)cx * (int64_t)a) ^ (uint64_t)((int64_t)cz * (int64_t)b) ^ world_seed;
    lcg_set_seed(st, s);
    return st;
}

// WorldCarver.carveEllipsoid (carver.c:165-214); the ellipsoid's cells are independent, so the
// warp's lanes take them in turn.  kind 0 = cave (floor level), 1 = canyon (width factors).
__device__ void carve_ellipsoid(CarveCtx &c, int kind, double floor_level, double x, double y, double z, double hr,
                                double vr) {
    const double reach = 16.0 + hr * 2.0;
    if (fabs(x - c.tmid_x) > reach || fabs(z - c.tmid_z) > reach) return;
    const int min_bx = c.tmin_x, min_bz = c.tmin_z;
    const int i0 = max(jfloor(x - hr) - min_bx - 1, 0);
    const int i1 = min(jfloor(x + hr) - min_bx, 15);
    const int k0 = max(jfloor(y - vr) - 1, -64 + 1);
    const int m0 = min(jfloor(y + vr) + 1, -64 + 384 - 1 - 7);
    const int n0 = max(jfloor(z - hr) - min_bz - 1, 0);
    const int o0 = min(jfloor(z + hr) - min_bz, 15);
    const int nxp = i1 - i0 + 1, nzp = o0 - n0 + 1, nyp = m0 - k0;
    if (nxp <= 0 || nzp <= 0 || nyp <= 0) return;
    const int lane = threadIdx.x & 31;
    // the normalised offsets depend on one coordinate each: divide once per row / column / level
    // (the same expressions, so the same doubles) instead of three times per block
    for (int q = lane; q < nxp; q += 32) c.fx[q] = ((double)(min_bx + i0 + q) + 0.5 - x) / hr;
    for (int q = lane; q < nzp; q += 32) c.fz[q] = ((double)(min_bz + n0 + q) + 0.5 - z) / hr;
    for (int q = lane; q < nyp; q += 32) c.fy[q] = ((double)(m0 - q) - 0.5 - y) / vr;
    __syncwarp();
    // the box's columns inside the horizontal ellipse (nx^2 + nz^2 < 1), compacted: the blocks of
    // the other columns are all skipped by that test
    int n_in = 0;
    for (int base = 0; base < nxp * nzp; base += 32) {
        const int q = base + lane;
        int pi = 0, si = 0;
        bool in = false;
        if (q < nxp * nzp) {
            pi = q / nzp;
            si = q - pi * nzp;
            in = c.fx[pi] * c.fx[pi] + c.fz[si] * c.fz[si] < 1.0;
        }
        const unsigned m = __ballot_sync(0xFFFFFFFFu, in);
        if (in) c.cols[n_in + __popc(m & ((1u << lane) - 1u))] = (uint16_t)((pi << 4) | si);
        n_in += __popc(m);
    }
    __syncwarp();
    const float inv_nyp = 1.0f / (float)nyp;
    for (int q = lane; q < n_in * nyp; q += 32) {
        int k = (int)((float)q * inv_nyp);   // q / nyp, corrected below (q < 2^17: one step suffices)
        if (k * nyp > q) k--;
        else if ((k + 1) * nyp <= q) k++;
        const int vi = q - k * nyp, pi = c.cols[k] >> 4, si = c.cols[k] & 15;
        const int p = i0 + pi, s = n0 + si, v = m0 - vi;
        const double nx = c.fx[pi];
        const double nz = c.fz[si];
        const double ny = c.fy[vi];
        bool skip;
        if (kind == 0) {
            skip = (ny <= floor_level) || (nx * nx + ny * ny + nz * nz) >= 1.0;
        } else {
            const int idx = v - (-64) - 1;
            skip = (nx * nx + nz * nz) * (double)c.width[idx] + ny * ny / 6.0 >= 1.0;
        }
        if (skip) continue;
        const int ci = carve_index(p, v, s);
        const uint32_t pre = c.J->states[ci];   // p2_block_at and p2_substance(.., 0.0), precomputed
        const uint32_t bit = 1u << (ci & 31);
        const uint32_t old = atomicOr(&c.mask[ci >> 5], bit);
        if (old & bit) continue;
        // carveBlock.  A block is written only after its mask bit is set, so an unmarked block
        // still holds its pre-carver state.
        const int st = (int)(pre & 15u);
        if (!(st == BS_SOLID || st == BS_WATER)) continue;
        int cs;
        if (v <= -56) {
            cs = BS_LAVA;
        } else {
            cs = (int)(pre >> 4);
            if (cs == BS_SOLID) continue;
        }
        c.cells[ci] = (uint8_t)cs;
    }
    __syncwarp();
}

__device__ float cave_thickness(uint64_t &r) {
    float f = lcg_float(r) * 2.0f + lcg_float(r);
    if (lcg_int(r, 10) == 0) {
        float a = lcg_float(r);
        float b = lcg_float(r);
        f = f * (a * b * 3.0f + 1.0f);
    }
    return f;
}

// createTunnel (carver.c:266-330).  A tunnel may split once into two thinner ones (thickness
// <= 1, so they never split again); the split tunnels are the kBranch = false instantiation,
// which keeps the call chain two levels deep without recursion.
template <bool kBranch>
__device__ __noinline__ void cave_tunnel(CarveCtx &c, double floor_level, uint64_t seed, double x, double y, double z,
                                         double d4, double d5, float thickness, float yaw, float pitch, int first_step,
                                         int total_steps, double y_scale) {
    const SinTab sn{c.sinq, c.sin_half_turn};
    const double tmid_x = c.tmid_x, tmid_z = c.tmid_z;
    uint64_t r;
    lcg_set_seed(r, seed);
    const int branch_step = lcg_int(r, total_steps / 2) + total_steps / 4;
    const bool wide = (lcg_int(r, 6) == 0);
    float f30 = 0.0f, f31 = 0.0f;
    for (int i = first_step; i < total_steps; i++) {
        const float ang = (float)i * 3.1415927f / (float)total_steps;
        const double radius = 1.5 + (double)(mc_sin(sn, (double)ang) * thickness);
        const double vert_base = radius * y_scale;
        const float cos_pitch = mc_cos(sn, (double)pitch);
        x += (double)(mc_cos(sn, (double)yaw) * cos_pitch);
        y += (double)mc_sin(sn, (double)pitch);
        z += (double)(mc_sin(sn, (double)yaw) * cos_pitch);
        pitch *= wide ? 0.92f : 0.7f;
        pitch += f31 * 0.1f;
        yaw += f30 * 0.1f;
        f31 *= 0.9f;
        f30 *= 0.75f;
        // six nextFloat, then (past the branch point) one nextInt(4): seven draws from r0
        const uint64_t r0 = r;
        f31 += (lcg_float_at(lcg_ahead<1>(r0)) - lcg_float_at(lcg_ahead<2>(r0))) * lcg_float_at(lcg_ahead<3>(r0)) *
               2.0f;
        f30 += (lcg_float_at(lcg_ahead<4>(r0)) - lcg_float_at(lcg_ahead<5>(r0))) * lcg_float_at(lcg_ahead<6>(r0)) *
               4.0f;
        if (kBranch && i == branch_step && thickness > 1.0f) {
            r = lcg_ahead<6>(r0);
            const uint64_t s1 = lcg_long(r);
            const float t1 = lcg_float(r) * 0.5f + 0.5f;
            cave_tunnel<false>(c, floor_level, s1, x, y, z, d4, d5, t1, yaw - 1.5707964f, pitch / 3.0f, i,
                               total_steps, 1.0);
            const uint64_t s2 = lcg_long(r);
            const float t2 = lcg_float(r) * 0.5f + 0.5f;
            cave_tunnel<false>(c, floor_level, s2, x, y, z, d4, d5, t2, yaw + 1.5707964f, pitch / 3.0f, i,
                               total_steps, 1.0);
            return;
        }
        r = lcg_ahead<7>(r0);
        if (lcg_int_pow2_at(r, 4) == 0) continue;
        {
            const double dx = x - tmid_x, dz = z - tmid_z;
            const double dy = (double)(total_steps - i);
            const double rr = (double)(thickness + 2.0f + 16.0f);
            if (!(dx * dx + dz * dz - dy * dy <= rr * rr)) return;
        }
        carve_ellipsoid(c, 0, floor_level, x, y, z, radius * d4, vert_base * d5);
    }
}

__device__ void cave_carve(CarveCtx &c, uint64_t &r, int ocx, int ocz, int y_hi) {
    const SinTab sn{c.sinq, c.sin_half_turn};
    const int i10 = lcg_int(r, lcg_int(r, lcg_int(r, 15) + 1) + 1);
    for (int k = 0; k < i10; k++) {
        const int lx = lcg_int(r, 16);
        const double x = (double)(ocx * 16 + lx);
        const int y = lcg_int(r, y_hi - (-56) + 1) + (-56);
        const int lz = lcg_int(r, 16);
        const double z = (double)(ocz * 16 + lz);
        const double hrm = (double)uniform_float(r, 0.7f, 1.4f);
        const double vrm = (double)uniform_float(r, 0.8f, 1.3f);
        const double floor_level = (double)uniform_float(r, -1.0f, -0.4f);
        int tunnels = 1;
        if (lcg_int(r, 4) == 0) {
            const double room_y_scale = (double)uniform_float(r, 0.1f, 0.9f);
            const float f28 = 1.0f + lcg_float(r) * 6.0f;
            const float sf = mc_sin(sn, 1.5707963705062866);
            const double d17 = 1.5 + (double)(sf * f28);
            const double d19 = d17 * room_y_scale;
            carve_ellipsoid(c, 0, floor_level, x + 1.0, (double)y, z, d17, d19);
            tunnels += lcg_int(r, 4);
        }
        for (int t = 0; t < tunnels; t++) {
            const float yaw = lcg_float(r) * 6.2831855f;
            const float pitch = (lcg_float(r) - 0.5f) / 4.0f;
            const float thick = cave_thickness(r);
            const int steps = 112 - lcg_int(r, 112 / 4);
            const uint64_t seed = lcg_long(r);
            cave_tunnel<true>(c, floor_level, seed, x, (double)y, z, hrm, vrm, thick, yaw, pitch, 0, steps, 1.0);
        }
    }
}

__device__ void canyon_carve(CarveCtx &c, uint64_t &r0, int ocx, int ocz) {
    const SinTab sn{c.sinq, c.sin_half_turn};
    const double tmid_x = c.tmid_x, tmid_z = c.tmid_z;
    const int lx = lcg_int(r0, 16);
    double x = (double)(ocx * 16 + lx);
    const int yi = lcg_int(r0, 67 - 10 + 1) + 10;
    const int lz = lcg_int(r0, 16);
    double z = (double)(ocz * 16 + lz);
    float yaw = lcg_float(r0) * 6.2831855f;
    float pitch = uniform_float(r0, -0.125f, 0.125f);
    const double y_scale = (double)3.0f;
    float thickness;
    {   // TrapezoidFloat(0, 6, plateau 2)
        const float d = 6.0f - 0.0f;
        const float e = (d - 2.0f) / 2.0f;
        const float f = d - e;
        const float a = lcg_float(r0) * f + 0.0f;
        thickness = a + lcg_float(r0) * e;
    }
    const float dist = uniform_float(r0, 0.75f, 1.0f);
    const int total_steps = (int)((float)112 * dist);
    const uint64_t seed = lcg_long(r0);
    // doCarve
    uint64_t r;
    lcg_set_seed(r, seed);
    const int lane = threadIdx.x & 31;
    {   // width factors: every lane draws the same sequence; lane 0 stores it
        float f = 1.0f;
        for (int i = 0; i < 384; i++) {
            if (i == 0 || lcg_int(r, 3) == 0) {
                const float a = lcg_float(r);
                const float b = lcg_float(r);
                f = 1.0f + a * b;
            }
            if (lane == 0) c.width[i] = f * f;
        }
        __syncwarp();
    }
    double y = (double)yi;
    float yaw_drift = 0.0f, pitch_drift = 0.0f;
    for (int i = 0; i < total_steps; i++) {
        // two uniform floats, six nextFloat and one nextInt(4): nine draws from r0
        const uint64_t r0 = r;
        const float ang = (float)i * 3.1415927f / (float)total_steps;
        double radius = 1.5 + (double)(mc_sin(sn, (double)ang) * thickness);
        double vert_radius = radius * y_scale;
        radius *= (double)(lcg_float_at(lcg_ahead<1>(r0)) * (1.0f - 0.75f) + 0.75f);
        {   // updateVerticalRadius
            const float f1 = (float)total_steps, f2 = (float)i;
            const float f7 = 1.0f - fabsf(0.5f - f2 / f1) * 2.0f;
            const float f8 = 0.0f + 1.0f * f7;
            const double base = (double)f8 * vert_radius;
            vert_radius = base * (double)(lcg_float_at(lcg_ahead<2>(r0)) * (1.0f - 0.75f) + 0.75f);
        }
        const float cos_pitch = mc_cos(sn, (double)pitch);
        const float sin_pitch = mc_sin(sn, (double)pitch);
        x += (double)(mc_cos(sn, (double)yaw) * cos_pitch);
        y += (double)sin_pitch;
        z += (double)(mc_sin(sn, (double)yaw) * cos_pitch);
        pitch *= 0.7f;
        pitch += pitch_drift * 0.05f;
        yaw += yaw_drift * 0.05f;
        pitch_drift *= 0.8f;
        yaw_drift *= 0.5f;
        pitch_drift += (lcg_float_at(lcg_ahead<3>(r0)) - lcg_float_at(lcg_ahead<4>(r0))) *
                       lcg_float_at(lcg_ahead<5>(r0)) * 2.0f;
        yaw_drift += (lcg_float_at(lcg_ahead<6>(r0)) - lcg_float_at(lcg_ahead<7>(r0))) *
                     lcg_float_at(lcg_ahead<8>(r0)) * 4.0f;
        r = lcg_ahead<9>(r0);
        if (lcg_int_pow2_at(r, 4) == 0) continue;
        {
            const double dx = x - tmid_x, dz = z - tmid_z;
            const double dy = (double)(total_steps - i);
            const double rr = (double)(thickness + 2.0f + 16.0f);
            if (!(dx * dx + dz * dz - dy * dy <= rr * rr)) return;
        }
        carve_ellipsoid(c, 1, 0.0, x, y, z, radius, vert_radius);
    }
}

// applyCarvers for the job's chunk (carver.c:482-523), one warp per chunk: a serial chain of tunnel
// walks and ellipsoids, whose blocks the lanes take in turn.  Shared memory holds the carve mask
// (12 KB), the sine quarter wave (64 KB) and small per-ellipsoid tables — 83 KB, two chunks per
// SM — while the cells stay in the job's global memory (L2 holds them).  The blocks' pre-carver
// states come from p2_states_kernel, which also clears the cells; they are not read as such while
// J.carved is 0, so they serve as the working copy.
__global__ void __launch_bounds__(kCarveThreads) p2_carve_kernel(const P2Tables *__restrict__ Tp,
                                                                 const P2World *__restrict__ worlds, P2Chunk *jobs) {
    __shared__ float width[384];
    __shared__ double fxs[16], fzs[16], fys[384];
    __shared__ uint16_t cols[256];
    __shared__ uint32_t mask[kMaskWords];   // blocks already carved
    extern __shared__ float4 sinq4[];       // Mth.SIN quarter wave, kSinQuarterPad floats
    P2Chunk &J = jobs[blockIdx.x];
    const P2World &W = worlds[J.world];
    uint8_t *cells = J.cells;   // all CV_UNCHANGED (p2_states_kernel)
    for (int q = threadIdx.x; q < kMaskWords; q += blockDim.x) mask[q] = 0u;
    const float4 *sinq_src = reinterpret_cast<const float4 *>(Tp->sin_quarter);
    for (int q = threadIdx.x; q < kSinQuarterPad / 4; q += blockDim.x) sinq4[q] = sinq_src[q];
    __syncwarp();
    CarveCtx c;
    c.sinq = reinterpret_cast<const float *>(sinq4);
    c.sin_half_turn = Tp->sin_half_turn;
    c.T = Tp;
    c.W = &W;
    c.J = &J;
    c.cells = cells;
    c.mask = mask;
    c.width = width;
    c.fx = fxs;
    c.fz = fzs;
    c.fy = fys;
    c.cols = cols;
    c.tmin_x = J.chunk_x * 16;
    c.tmin_z = J.chunk_z * 16;
    c.tmid_x = (double)(c.tmin_x + 8);
    c.tmid_z = (double)(c.tmin_z + 8);
    // the (dx, dz, carver) triples in order, dx outer: each lane tests one of 32 at a time for
    // the carver's start probability, and the warp runs the ones that start, in order
    constexpr int kTriples = 17 * 17 * 3;
    const int lane = threadIdx.x & 31;
    for (int base = 0; base < kTriples; base += 32) {
        const int q = base + lane;
        bool starts = false;
        uint64_t rq = 0;
        if (q < kTriples) {
            const int ci = q % 3, dx = q / 51 - 8, dz = (q / 3) % 17 - 8;
            const float prob = ci == 0 ? 0.15f : (ci == 1 ? 0.07f : 0.01f);
            rq = large_feature_state(W.seed + (uint64_t)ci, J.chunk_x + dx, J.chunk_z + dz);
            starts = lcg_float(rq) <= prob;
        }
        unsigned pending = __ballot_sync(0xFFFFFFFFu, starts);
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1;
            uint64_t r = __shfl_sync(0xFFFFFFFFu, rq, src);
            const int t = base + src, ci = t % 3;
            const int ox = J.chunk_x + t / 51 - 8, oz = J.chunk_z + (t / 3) % 17 - 8;
            if (ci == 1) cave_carve(c, r, ox, oz, 47);
            else if (ci == 0) cave_carve(c, r, ox, oz, 180);
            else canyon_carve(c, r, ox, oz);
        }
    }
    __syncwarp();
    __threadfence_block();
    if (threadIdx.x == 0) J.carved = 1;
}

// ------------------------------------------------------------------------------------
// Biome gate (biome.c) and the verdict (eval.c)
// ------------------------------------------------------------------------------------
__device__ int64_t tree_dist(const BiomeTree &g, int i, const int64_t np[6]) {
    int64_t ds = 0;
    for (int k = 0; k < 6; k++) {
        int64_t d = np[k] - g.range[12 * i + 2 * k + 1], e = (int64_t)g.range[12 * i + 2 * k] - np[k];
        d = d > 0 ? d : (e > 0 ? e : 0);
        ds += d * d;
    }
    return ds;
}

// Climate.RTree.SubTree.search (biome.c:35-48) with an explicit stack instead of recursion:
// a frame is one inner node scanning its children (k-th child at index c) with the best leaf
// so far.  The host checks at upload that no tree nests deeper than kTreeDepth.
__device__ int tree_search(const BiomeTree &g, const int64_t np[6]) {
    int fnode[kTreeDepth], fk[kTreeDepth], fc[kTreeDepth], fres[kTreeDepth];
    int64_t fbest[kTreeDepth], fd[kTreeDepth];
    if (g.kids[0] == 0) return 0;
    int sp = 0;
    fnode[0] = 0;
    fk[0] = 0;
    fc[0] = 1;
    fres[0] = -1;
    fbest[0] = 0x7FFFFFFFFFFFFFFFLL;
    int ret = -1;
    bool returning = false;
    for (;;) {
        if (returning) {   // the search below child fc[sp] returned leaf `ret`
            const int c = fc[sp];
            const int64_t d2 = (ret == c) ? fd[sp] : tree_dist(g, ret, np);
            if (fbest[sp] > d2) {
                fbest[sp] = d2;
                fres[sp] = ret;
            }
            fk[sp]++;
            fc[sp] = g.end[c];
            returning = false;
        }
        if (fk[sp] < g.kids[fnode[sp]]) {
            const int c = fc[sp];
            const int64_t d = tree_dist(g, c, np);
            if (fbest[sp] > d) {
                fd[sp] = d;
                if (g.kids[c] == 0) {   // a leaf returns itself
                    ret = c;
                    returning = true;
                    continue;
                }
                if (sp + 1 >= kTreeDepth) return -1;
                const int leaf = fres[sp];
                sp++;
                fnode[sp] = c;
                fk[sp] = 0;
                fc[sp] = c + 1;
                fres[sp] = leaf;
                fbest[sp] = leaf < 0 ? 0x7FFFFFFFFFFFFFFFLL : tree_dist(g, leaf, np);
                continue;
            }
            fk[sp]++;
            fc[sp] = g.end[c];
            continue;
        }
        ret = fres[sp];
        if (sp == 0) return ret;
        sp--;
        returning = true;
    }
}

// The biome lysh_swamp_hut_biome_ok reports at a chunk's middle column (mid_x, mid_z) when the
// surface there is at y + 1 (biome.c:94-156): the six climate parameters at quart
// (mid_x >> 2, y >> 2, mid_z >> 2), quantised through float, and the nearest leaf of the tree.
// The offset spline is evaluated at the same quart column (the reference asks for block
// (qx * 4, qz * 4) >> 2, which is qx, qz again).
// The y-independent half of the six climate parameters at block column (mid_x, mid_z).
struct ColumnClimate {
    double temperature, humidity, c, e, w, offset;
};
__device__ ColumnClimate p2_column_climate(const P2Tables &T, const P2World &W, int mid_x, int mid_z) {
    TerrainInfo ti;
    p2_terrain(T, W, mid_x >> 2, mid_z >> 2, ti);
    ColumnClimate cc;
    cc.temperature = p2_dbl(T, W, Q_TEMPERATURE, ti.sx, 0.0, ti.sz);
    cc.humidity = p2_dbl(T, W, Q_VEGETATION, ti.sx, 0.0, ti.sz);
    double factor;
    p2_offset_factor(T, ti, cc.offset, factor);
    cc.c = ti.c;
    cc.e = ti.e;
    cc.w = ti.w;
    return cc;
}

// The climate point at height y (depth from the column's offset) and the R-tree's biome.
__device__ int p2_biome_at_y(const P2Tables &T, int tree, const ColumnClimate &cc, int y, int64_t np[6]) {
    const int qy = y >> 2;
    const double yq = (double)(qy * 4);
    const double depth = mc_lerp(mc_clamp((yq - -64.0) / (320.0 - -64.0), 0.0, 1.0), 1.5, -1.5) + cc.offset;
    np[0] = (int64_t)((float)cc.temperature * 10000.0f);
    np[1] = (int64_t)((float)cc.humidity * 10000.0f);
    np[2] = (int64_t)((float)cc.c * 10000.0f);
    np[3] = (int64_t)((float)cc.e * 10000.0f);
    np[4] = (int64_t)((float)depth * 10000.0f);
    np[5] = (int64_t)((float)cc.w * 10000.0f);
    const BiomeTree &g = T.trees[tree];
    const int leaf = tree_search(g, np);
    return leaf >= 0 ? g.biome[leaf] : -1;
}

__device__ int p2_biome_params(const P2Tables &T, const P2World &W, int tree, int mid_x, int mid_z, int y,
                               int64_t np[6]) {
    return p2_biome_at_y(T, tree, p2_column_climate(T, W, mid_x, mid_z), y, np);
}

__device__ __forceinline__ int64_t floor_div16(int64_t v) { return v >= 0 ? v / 16 : -((-v + 15) / 16); }

// biome_map's raster (engine/tools/mineshaft/biome_map.c:105-127): cell (i, j) samples ss x ss
// points, each the biome at the middle of the chunk holding it with the surface at y + 1; the
// first id to reach the highest count wins, and a swamp that fills a quarter of the samples wins.
__global__ void __launch_bounds__(128) p2_biome_map_kernel(const P2Tables *__restrict__ Tp, const P2World *__restrict__ worlds,
                                                           int tree, int64_t x0, int64_t z0, int w, int h, int step,
                                                           int ss, int y, uint8_t *out) {
    const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= (int64_t)w * h) return;
    const P2Tables &T = *Tp;
    const P2World &W = worlds[0];
    const int i = (int)(cell % w), j = (int)(cell / w);
    uint8_t ids[16];
    int n = 0;
    for (int b = 0; b < ss; b++) {
        const int64_t Z = z0 + (int64_t)j * step + ((2LL * b + 1) * step) / (2LL * ss);
        for (int a = 0; a < ss; a++) {
            const int64_t X = x0 + (int64_t)i * step + ((2LL * a + 1) * step) / (2LL * ss);
            const int cx = (int)floor_div16(X), cz = (int)floor_div16(Z);
            int64_t np[6];
            ids[n++] = (uint8_t)(p2_biome_params(T, W, tree, cx * 16 + 8, cz * 16 + 8, y, np) & 0xFF);
        }
    }
    int best = -1, best_n = 0, swamps = 0;
    for (int k = 0; k < n; k++) {
        int c = 0;
        for (int q = 0; q <= k; q++) c += ids[q] == ids[k];
        if (c > best_n) {
            best_n = c;
            best = ids[k];
        }
        swamps += ids[k] == 6;
    }
    if (swamps * 4 >= n && swamps > 0) best = 6;
    out[cell] = (uint8_t)best;
}

// biome_map --stdin's first pass (biome_map.c:38-52): the biome at each chunk's middle with the
// surface at y + 1 for y = 40, 48, ..., 80; all swamp or no swamp settles it (the answer is the
// swamp, or the y = 64 biome), a disagreement needs the real surface height (need[i] = 1).
__global__ void __launch_bounds__(128) p2_biome_chunks_kernel(const P2Tables *__restrict__ Tp,
                                                              const P2World *__restrict__ worlds, int tree,
                                                              const int32_t *__restrict__ cx, const int32_t *__restrict__ cz,
                                                              int n, uint8_t *out, uint8_t *need) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const P2Tables &T = *Tp;
    const P2World &W = worlds[0];
    int swamps = 0, first = 0;
    for (int q = 0; q < 6; q++) {
        int64_t np[6];
        const int id = p2_biome_params(T, W, tree, cx[k] * 16 + 8, cz[k] * 16 + 8, 40 + 8 * q, np) & 0xFF;
        if (q == 3) first = id;
        swamps += id == 6;
    }
    const bool settled = swamps == 0 || swamps == 6;
    out[k] = (uint8_t)(settled ? (swamps ? 6 : first) : 0);
    need[k] = settled ? 0 : 1;
}

// The biome winner of the R-tree `tree` at column (x, z) with first occupied height y, in world
// pts[4k] (biome_at: lysh_swamp_hut_biome_ok with a constant height callback, biome.c:94-156).
// pts holds (world, x, z, y) per point; x and z are the column's middle blocks.
__global__ void __launch_bounds__(128) p2_biome_points_kernel(const P2Tables *__restrict__ Tp,
                                                              const P2World *__restrict__ worlds, int tree,
                                                              const int32_t *__restrict__ pts, int n,
                                                              int32_t *__restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int64_t np[6];
    out[k] = p2_biome_params(*Tp, worlds[pts[4 * k]], tree, pts[4 * k + 1], pts[4 * k + 2], pts[4 * k + 3], np);
}

constexpr int kFinishThreads = 96;   // 63 footprint columns, the chunk centre, the centre's climate

__global__ void __launch_bounds__(kFinishThreads) p2_finish_kernel(const P2Tables *__restrict__ Tp,
                                                                   const P2World *__restrict__ worlds,
                                                                   const P2Chunk *__restrict__ jobs,
                                                                   const P2Hut *__restrict__ huts, int tree,
                                                                   P2Result *out) {
    __shared__ int pre_h[64], post_h[64], wet[64];
    __shared__ int size_x, size_z;
    __shared__ ColumnClimate centre;
    const P2Tables &T = *Tp;
    const P2Hut H = huts[blockIdx.x];
    const P2Chunk &J = jobs[H.job];
    const P2World &W = worlds[J.world];
    P2Result &R = out[blockIdx.x];
    const int t = threadIdx.x;
    if (t == 0) {
        const int dir = hut_dir(W.seed, H.hut_x, H.hut_z);
        const int axis_z = (dir == 0 || dir == 2);
        size_x = axis_z ? 7 : 9;
        size_z = axis_z ? 9 : 7;
        R.hut_x = H.hut_x;
        R.hut_z = H.hut_z;
        R.rx = floor_div(H.hut_x, 32);
        R.rz = floor_div(H.hut_z, 32);
        R.dir = dir;
        R.axis_z = axis_z;
        R.size_x = size_x;
        R.size_z = size_z;
    }
    __syncthreads();
    // footprint column t (dx outer, dz inner), and the chunk-centre column as t == 63
    if (t < 63) {
        const int dx = t / size_z, dz = t % size_z;
        const int x = H.hut_x + dx, z = H.hut_z + dz;
        int level, type;
        p2_compute_fluid(T, W, &J, x, 62, z, level, type);
        wet[t] = (type == BS_WATER && 62 < level) ? 1 : 0;
        pre_h[t] = p2_height(T, W, J, x, z, false);
        post_h[t] = p2_height(T, W, J, x, z, true);
    } else if (t == 63) {
        const int mid_x = (H.hut_x >> 4) * 16 + 8, mid_z = (H.hut_z >> 4) * 16 + 8;
        pre_h[63] = p2_height(T, W, J, mid_x, mid_z, false);
    } else if (t == 64) {   // the y-independent climate at the chunk centre, beside the column work
        centre = p2_column_climate(T, W, (H.hut_x >> 4) * 16 + 8, (H.hut_z >> 4) * 16 + 8);
    }
    __syncthreads();
    if (t != 0) return;
    // biome gate at the chunk centre (biome.c:94-156)
    {
        const int mid_x = (H.hut_x >> 4) * 16 + 8, mid_z = (H.hut_z >> 4) * 16 + 8;
        const int y = pre_h[63] - 1;
        int64_t np[6];
        const int winner = p2_biome_at_y(T, tree, centre, y, np);
        for (int a = 0; a < 6; a++) R.biome_t[a] = np[a];
        R.biome_qx = mid_x >> 2;
        R.biome_qy = y >> 2;
        R.biome_qz = mid_z >> 2;
        R.biome_occ_y = y;
        R.biome_winner = winner;
        R.biome_ok = winner == 6 ? 1 : 0;
    }
    int nwet = 0;
    for (int k = 0; k < 63; k++) nwet += wet[k];
    R.wet_columns = nwet;
    R.flooded = nwet == 63;
    R.all_dry = nwet == 0;
    long long sum = 0;
    bool carve_skipped = false;
    if (R.flooded) {
        bool blocked = false;
        long long sum_pre = 0;
        for (int k = 0; k < 63 && !blocked; k++) {
            sum_pre += pre_h[k];
            if (pre_h[k] - 1 >= 64) blocked = true;
        }
        if (!blocked) {
            sum = sum_pre;
            carve_skipped = true;
        }
    }
    if (!carve_skipped)
        for (int k = 0; k < 63; k++) sum += post_h[k];
    R.sum_h = sum;
    R.avg_y = (int)(sum / 63);
    if (!R.biome_ok) {
        R.ok = 0;
        R.reject = 3;
    } else if (R.flooded) {
        R.ok = 0;
        R.reject = 2;
    } else if (R.avg_y > H.max_y) {
        R.ok = 0;
        R.reject = 1;
    } else {
        R.ok = 1;
        R.reject = 0;
    }
}

// ------------------------------------------------------------------------------------
// Point probes
// ------------------------------------------------------------------------------------
__global__ void p2_probe_kernel(const P2Tables *__restrict__ Tp, const P2World *__restrict__ worlds,
                                const P2Chunk *__restrict__ jobs, const int32_t *__restrict__ pts, int n, int kind,
                                double *out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const P2Tables &T = *Tp;
    const int32_t *p = pts + 5 * q;
    const P2World &W = worlds[p[0]];
    const int x = p[1], y = p[2], z = p[3], job = p[4];
    double v = 0.0;
    switch (kind) {
        case PR_BASE_NOISE: v = p2_blended(T, W, x, y, z); break;
        case PR_DENSITY_RAW: v = p2_density_raw(T, W, x, y, z); break;
        case PR_COLUMN_TOP: v = (double)p2_column_top(T, W, x, z); break;
        case PR_CONTINENTALNESS:
        case PR_EROSION:
        case PR_WEIRDNESS: {
            TerrainInfo ti;
            p2_terrain(T, W, x >> 2, z >> 2, ti);
            v = kind == PR_CONTINENTALNESS ? ti.c : (kind == PR_EROSION ? ti.e : ti.w);
            break;
        }
        case PR_OFFSET_261:
        case PR_FACTOR_261:
        case PR_PEAKS_261: {
            TerrainInfo ti;
            p2_terrain(T, W, x >> 2, z >> 2, ti);
            const TerrainPoint tp = p2_point_261(T, ti);
            v = kind == PR_OFFSET_261 ? (double)tp.offset : (kind == PR_FACTOR_261 ? (double)tp.factor : (double)tp.peaks);
            break;
        }
        case PR_FLUID: {
            int level, type;
            p2_compute_fluid(T, W, nullptr, x, y, z, level, type);
            v = (double)level * 4.0 + (double)type;
            break;
        }
        case PR_DENSITY: v = p2_density_at(T, W, jobs[job], x, y, z); break;
        case PR_BLOCK: v = (double)p2_block_at(T, W, jobs[job], x, y, z); break;
        case PR_HEIGHT_PRE: v = (double)p2_height(T, W, jobs[job], x, z, false); break;
        case PR_HEIGHT: v = (double)p2_height(T, W, jobs[job], x, z, true); break;
        case PR_GRID_MAIN: {
            const P2Chunk &J = jobs[job];
            const int c = ((x >> 2) - J.chunk_x * 4) * 5 + ((z >> 2) - J.chunk_z * 4);
            const int i = (y + 64) >> 3;
            v = (c >= 0 && c < kGridCols && i >= 0 && i < kGridYs) ? J.main[c][i] : -1.0e300;
            break;
        }
        default: break;
    }
    out[q] = v;
}

}  // namespace

// ------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------
void p2_launch_legacy(const P2Tables *T, P2World *worlds, int n_worlds, cudaStream_t s) {
    if (n_worlds > 0) p2_legacy_kernel<<<n_worlds, 64, 0, s>>>(T, worlds);
}

void p2_launch_build(const P2Tables *T, P2World *worlds, int n_worlds, cudaStream_t s) {
    const dim3 grid((kWorldSlotsMax + kBuildThreads - 1) / kBuildThreads, n_worlds);
    p2_build_kernel<<<grid, kBuildThreads, 0, s>>>(T, worlds);
}

void p2_launch_grid(const P2Tables *T, const P2World *worlds, P2Chunk *jobs, int n_jobs, cudaStream_t s) {
    p2_grid_kernel<<<dim3(n_jobs, 5), kGridThreads, 0, s>>>(T, worlds, jobs);
}

void p2_launch_aquifer(const P2Tables *T, const P2World *worlds, P2Chunk *jobs, int n_jobs, cudaStream_t s) {
    p2_tops_kernel<<<dim3(n_jobs, 5), kAqThreads, 0, s>>>(T, worlds, jobs);
    p2_aquifer_kernel<<<dim3(n_jobs, 3), kAqThreads, 0, s>>>(T, worlds, jobs);
}

void p2_launch_states(const P2Tables *T, const P2World *worlds, P2Chunk *jobs, int n_jobs, cudaStream_t s) {
    p2_states_kernel<<<dim3(kCarveCells / 256, n_jobs), 256, 0, s>>>(T, worlds, jobs);
}

void p2_launch_carve(const P2Tables *T, const P2World *worlds, P2Chunk *jobs, int n_jobs, cudaStream_t s) {
    static_assert(kSinQuarterPad % 4 == 0, "the quarter wave is copied as float4");
    constexpr int smem = kSinQuarterPad * (int)sizeof(float);
    cudaFuncSetAttribute(p2_carve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    p2_carve_kernel<<<n_jobs, kCarveThreads, smem, s>>>(T, worlds, jobs);
}

void p2_launch_biome_map(const P2Tables *T, const P2World *worlds, int tree, int64_t x0, int64_t z0, int w, int h,
                         int step, int ss, int y, uint8_t *out, cudaStream_t s) {
    const int64_t cells = (int64_t)w * h;
    p2_biome_map_kernel<<<(unsigned)((cells + 127) / 128), 128, 0, s>>>(T, worlds, tree, x0, z0, w, h, step, ss, y, out);
}

void p2_launch_biome_chunks(const P2Tables *T, const P2World *worlds, int tree, const int32_t *cx, const int32_t *cz,
                            int n, uint8_t *out, uint8_t *need, cudaStream_t s) {
    p2_biome_chunks_kernel<<<(n + 127) / 128, 128, 0, s>>>(T, worlds, tree, cx, cz, n, out, need);
}

void p2_launch_biome_points(const P2Tables *T, const P2World *worlds, int tree, const int32_t *pts, int n,
                            int32_t *out, cudaStream_t s) {
    if (n > 0) p2_biome_points_kernel<<<(n + 127) / 128, 128, 0, s>>>(T, worlds, tree, pts, n, out);
}

void p2_launch_finish(const P2Tables *T, const P2World *worlds, const P2Chunk *jobs, const P2Hut *huts, int n_huts,
                      int tree, P2Result *out, cudaStream_t s) {
    p2_finish_kernel<<<n_huts, kFinishThreads, 0, s>>>(T, worlds, jobs, huts, tree, out);
}

void p2_launch_probe(const P2Tables *T, const P2World *worlds, const P2Chunk *jobs, const int32_t *pts, int n_pts,
                     int kind, double *out, cudaStream_t s) {
    p2_probe_kernel<<<(n_pts + 127) / 128, 128, 0, s>>>(T, worlds, jobs, pts, n_pts, kind, out);
}

}  // namespace wg
