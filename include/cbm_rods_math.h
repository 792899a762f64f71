/*
 * cbm_rods_math.h — the contact force of the rods2D model, for the device and
 * the host alike (inline, no exports).
 *
 * rodForces (src/models/rods.jl:21-59) and its geometry in CBMMetrics
 * (src/metrics.jl: intersection2lines :137-152, point2line :162-170,
 * pointInsideRod :182-190, rodIntersection :202-246), expression by
 * expression (rodIntersection computes the projections its cases share once;
 * see there).  Definitions of this build where Julia's arithmetic is not
 * reproduced:
 *  - cos and sin: the library's own series of cbm_rng.h, on theta/(2 pi)
 *    reduced to [0, 1), so host and device give the same bits;
 *  - delta^1.5 = delta sqrt(delta) and delta^0.5 = sqrt(delta);
 *  - in Float32 every operation and constant is Float32 (Julia would promote
 *    the Float64 literals 0.99, 1e-6, 1e-7, 1e-8 and what follows them).
 * Builds keep every a*b+c as two rounded operations (-fmad=false on the
 * device, -ffp-contract=off on the host).
 */
#ifndef CBM_RODS_MATH_H
#define CBM_RODS_MATH_H

#include <math.h>

#include "cbm_rng.h"

/* cos and sin of an angle in radians */
template <typename T>
CBM_HD void cbm_rod_cossin(T th, T* c, T* s) {
  T w = th * (T)0.15915494309189535; /* 1 / (2 pi) */
  w = w - floor(w);
  if (w >= (T)1) w = w - (T)1;
  if (sizeof(T) == 8) {
    double cc, ss;
    cbm_cossin_turns_f64((double)w, &cc, &ss);
    *c = (T)cc;
    *s = (T)ss;
  } else {
    float cc, ss;
    cbm_cossin_turns_f32((float)w, &cc, &ss);
    *c = (T)cc;
    *s = (T)ss;
  }
}

/* Julia's min / max of two floats: NaN wins, -0 < +0 */
template <typename T>
CBM_HD T cbm_jl_min(T a, T b) {
  if (a != a || b != b) return a + b;
  return (b < a || (b == a && signbit(b) && !signbit(a))) ? b : a;
}
template <typename T>
CBM_HD T cbm_jl_max(T a, T b) {
  if (a != a || b != b) return a + b;
  return (b > a || (b == a && !signbit(b) && signbit(a))) ? b : a;
}

/* A rod: centre, direction (cos, sin of theta), length */
template <typename T>
struct CbmRodGeom {
  T x, y, c, s, l;
};

/* point2line(x1, y1, x2, y2, theta2): the point of the line through (x2, y2)
 * along theta2 closest to (x1, y1) */
template <typename T>
CBM_HD void cbm_point2line(T x1, T y1, const CbmRodGeom<T>& r, T* ox, T* oy) {
  const T cx = r.x - x1, cy = r.y - y1;
  const T t = r.s * cx - r.c * cy;
  *ox = t * r.s + x1;
  *oy = -t * r.c + y1;
}

/* pointInsideRod(x1, y1, l1, theta1, px, py, separation) */
template <typename T>
CBM_HD void cbm_point_inside_rod(const CbmRodGeom<T>& r, T px, T py, T sep, T* ox, T* oy) {
  const T ex = r.x - px, ey = r.y - py;
  const T di = cbm_jl_max(sqrt(ex * ex + ey * ey), (T)0.00000001);
  const T dxi = (px - r.x) / di, dyi = (py - r.y) / di;
  const T a = sep * cbm_jl_min(di, r.l / (T)2);
  *ox = a * dxi + r.x;
  *oy = a * dyi + r.y;
}

/* intersection2lines(x1, y1, theta1, x2, y2, theta2) */
template <typename T>
CBM_HD void cbm_intersection2lines(const CbmRodGeom<T>& a, const CbmRodGeom<T>& b, T* px,
                                   T* py) {
  const T cx = a.x - b.x, cy = a.y - b.y;
  const T norm = a.c * b.s - a.s * b.c;
  if (fabs(norm) > (T)0.0000001) {
    const T scale = (-b.s * cx + b.c * cy) / norm;
    *px = scale * a.c + a.x;
    *py = scale * a.s + a.y;
  } else {
    *px = (a.x + b.x) / (T)2;
    *py = (a.y + b.y) / (T)2;
  }
}

/* rodIntersection(x1, y1, l1, theta1, x2, y2, l2, theta2; separation = 0.99):
 * the closest virtual spheres of the two rods.  The four cases of rods that
 * are not parallel use four projections of the lines' intersection p:
 * P1 = pointInsideRod(rod 1, p), P2 = pointInsideRod(rod 2, p),
 * S1 = point2line(P2 onto rod 1) and S2 = point2line(P1 onto rod 2).  They
 * are computed once, with the reference's expressions, and each case takes
 * its own (so lanes of one warp in different cases share the work instead of
 * running each case's projections in turn); the values are those of the
 * reference's case-by-case statements. */
template <typename T>
CBM_HD void cbm_rod_intersection(const CbmRodGeom<T>& a, const CbmRodGeom<T>& b, T* x1a, T* y1a,
                                 T* x2a, T* y2a) {
  const T sep = (T)0.99;
  T px, py;
  cbm_intersection2lines(a, b, &px, &py);
  T ex = a.x - px, ey = a.y - py;
  const T di = sqrt(ex * ex + ey * ey);
  ex = b.x - px;
  ey = b.y - py;
  const T dj = sqrt(ex * ex + ey * ey);
  const T norm = a.c * b.s - a.s * b.c;
  const T h1 = a.l / (T)2, h2 = b.l / (T)2;
  if (fabs(norm) < (T)0.000001) {  // parallel: projections of p onto each line
    T qx, qy;
    cbm_point2line(px, py, a, &qx, &qy);
    cbm_point_inside_rod(a, qx, qy, sep, x1a, y1a);
    cbm_point2line(px, py, b, &qx, &qy);
    cbm_point_inside_rod(b, qx, qy, sep, x2a, y2a);
    return;
  }
  T p1x, p1y, p2x, p2y, s1x, s1y, s2x, s2y;
  cbm_point_inside_rod(a, px, py, sep, &p1x, &p1y);
  cbm_point_inside_rod(b, px, py, sep, &p2x, &p2y);
  cbm_point2line(p2x, p2y, a, &s1x, &s1y);
  cbm_point2line(p1x, p1y, b, &s2x, &s2y);
  if (di <= h1 && dj <= h2) {  // p inside both rods
    *x1a = p1x;
    *y1a = p1y;
    *x2a = p2x;
    *y2a = p2y;
  } else if (di <= h1 && dj > h2) {  // p inside rod 1 only
    *x2a = p2x;
    *y2a = p2y;
    *x1a = s1x;
    *y1a = s1y;
  } else if (di > h1 && dj <= h2) {  // p inside rod 2 only
    *x1a = p1x;
    *y1a = p1y;
    *x2a = s2x;
    *y2a = s2y;
  } else {  // inside neither (or a comparison with NaN)
    *x2a = p2x;
    *y2a = p2y;
    *x1a = s1x;
    *y1a = s1y;
    ex = a.x - s1x;
    ey = a.y - s1y;
    if (sqrt(ex * ex + ey * ey) > h1) {
      *x1a = p1x;
      *y1a = p1y;
      ex = b.x - s2x;
      ey = b.y - s2y;
      if (sqrt(ex * ex + ey * ey) < h2) {
        *x2a = s2x;
        *y2a = s2y;
      }
    }
  }
}

/* Model constants of rodForces */
template <typename T>
struct CbmRodCoef {
  T kn, gn, gt, mucc;
};

/* rodForces: the force (fx, fy) and torque w on rod 1 from rod 2, with rod 1's
 * diameter d1, mass m1 and velocity (vx1, vy1); returns false without contact */
template <typename T>
CBM_HD bool cbm_rod_forces(const CbmRodGeom<T>& a, T d1, T vx1, T vy1, T m1,
                           const CbmRodGeom<T>& b, T d2, T vx2, T vy2, const CbmRodCoef<T>& k,
                           T* fx, T* fy, T* w) {
  T xi, yi, xj, yj;
  cbm_rod_intersection(a, b, &xi, &yi, &xj, &yj);
  const T ex = xi - xj, ey = yi - yj;
  const T rij = sqrt(ex * ex + ey * ey);
  if (!(rij > (T)0 && rij < (d1 + d2) / (T)2)) return false;
  const T delta = d1 - rij;
  const T me = m1 / (T)2;
  const T nx = (xi - xj) / rij, ny = (yi - yj) / rij;
  const T vijx = vx1 - vx2, vijy = vy1 - vy2;
  const T vn = nx * vijx + ny * vijy;
  const T sd = sqrt(delta);
  const T fn = k.kn * (delta * sd) - ((k.gn * me) * delta) * vn;
  const T ft = -cbm_jl_min((k.gt * me) * sd, k.mucc * fn);
  *fx = fn * nx + ft * (vijx - vn * nx);
  *fy = fn * ny + ft * (vijy - vn * ny);
  *w = (xi - a.x) * (*fy) - (yi - a.y) * (*fx);
  return true;
}

#endif /* CBM_RODS_MATH_H */
