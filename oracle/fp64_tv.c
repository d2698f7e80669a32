/* FP64 restatement of the TV proximal step (FGP on the dual of isotropic TV with a non-negativity
 * constraint), used by oracle/fp64.py to run the reference's reconstruction in double precision.
 *
 * TEST INFRASTRUCTURE: the error of a float32 result against this double-precision run is a
 * reported figure (how far float32 arithmetic strays from exact arithmetic of the same algorithm),
 * never the product path.
 *
 * The iteration is the reference's cpu::tv_prox (src/cpu/tv.cpp:7-44) with the shared formulas of
 * src/common.hpp:107-153: warm-started dual p, r = p, t = 1; per step x = max(b - lam L(r), 0),
 * gradient g = x - x[next] along each axis (zero on the last plane / row / column), q = r + g/(12 lam),
 * projection of q onto the unit ball, FISTA momentum (t - 1)/t_next on the dual; at the end
 * x = max(b - lam L(p), 0). L(q) = -div q accumulated in the same order as tv_adjoint. All in double,
 * two passes over the volume per step (primal, then dual), OpenMP over planes.
 *
 * Build: gcc -O2 -fopenmp -shared -fPIC (oracle/fp64.py does it). */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static double adjoint_at(const double* qz, const double* qy, const double* qx, int nz, int ny, int nx, int z, int y,
                         int x) {
  const size_t nxy = (size_t)nx * ny;
  const size_t i = (size_t)z * nxy + (size_t)y * nx + x;
  double s = 0.0;
  if (z < nz - 1) s += qz[i];
  if (z > 0) s -= qz[i - nxy];
  if (y < ny - 1) s += qy[i];
  if (y > 0) s -= qy[i - nx];
  if (x < nx - 1) s += qx[i];
  if (x > 0) s -= qx[i - 1];
  return s;
}

static void primal(const double* b, const double* qz, const double* qy, const double* qx, int nz, int ny, int nx,
                   double lam, double* out) {
  const size_t nxy = (size_t)nx * ny;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z) {
    for (int y = 0; y < ny; ++y) {
      for (int x = 0; x < nx; ++x) {
        const size_t i = (size_t)z * nxy + (size_t)y * nx + x;
        const double v = b[i] - lam * adjoint_at(qz, qy, qx, nz, ny, nx, z, y, x);
        out[i] = v > 0.0 ? v : 0.0;
      }
    }
  }
}

/* b: (nz, ny, nx); p: 3 volumes (z, y, x components), updated in place (warm start); x: output. */
int fp64_tv_prox(const double* b, double* p, int nz, int ny, int nx, double lam, int inner, double* x) {
  if (nz < 1 || ny < 1 || nx < 1 || !(lam > 0.0) || inner < 0) return 1;
  const size_t v = (size_t)nz * ny * nx;
  const size_t nxy = (size_t)nx * ny;
  double* r = (double*)malloc(3 * v * sizeof(double));
  if (!r) return 2;
  for (size_t i = 0; i < 3 * v; ++i) r[i] = p[i];
  double* pz = p;
  double* py = p + v;
  double* px = p + 2 * v;
  double* rz = r;
  double* ry = r + v;
  double* rx = r + 2 * v;
  const double step = 1.0 / (12.0 * lam);
  double t = 1.0;
  for (int k = 0; k < inner; ++k) {
    primal(b, rz, ry, rx, nz, ny, nx, lam, x);
    const double t_next = 0.5 * (1.0 + sqrt(1.0 + 4.0 * t * t));
    const double m = (t - 1.0) / t_next;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z) {
      for (int y = 0; y < ny; ++y) {
        for (int xx = 0; xx < nx; ++xx) {
          const size_t i = (size_t)z * nxy + (size_t)y * nx + xx;
          const double c = x[i];
          const double gz = z < nz - 1 ? c - x[i + nxy] : 0.0;
          const double gy = y < ny - 1 ? c - x[i + nx] : 0.0;
          const double gx = xx < nx - 1 ? c - x[i + 1] : 0.0;
          const double qz = rz[i] + step * gz;
          const double qy = ry[i] + step * gy;
          const double qx = rx[i] + step * gx;
          const double norm2 = qz * qz + qy * qy + qx * qx;
          const double s = norm2 > 1.0 ? 1.0 / sqrt(norm2) : 1.0;
          const double nz_ = qz * s, ny_ = qy * s, nx_ = qx * s;
          rz[i] = nz_ + m * (nz_ - pz[i]);
          ry[i] = ny_ + m * (ny_ - py[i]);
          rx[i] = nx_ + m * (nx_ - px[i]);
          pz[i] = nz_;
          py[i] = ny_;
          px[i] = nx_;
        }
      }
    }
    t = t_next;
  }
  primal(b, pz, py, px, nz, ny, nx, lam, x);
  free(r);
  return 0;
}

int fp64_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
