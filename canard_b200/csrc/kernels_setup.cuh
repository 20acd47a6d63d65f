// FP64-only device kernels of set-up and of the state bookkeeping: grid
// metrics, Jacobian, face normals, the qo copy, junction averaging and the
// FP32 copies of the metrics. Included by the FP64 translation unit only.
#pragma once
#include "kernels.cuh"

namespace canard {

__global__ void k_copy5(const BlockDev* __restrict__ bd) {  // qo = qa
  FOR_POINTS(bd[blockIdx.y]) {
    const long long n = B.npad;
#pragma unroll
    for (int c = 0; c < 5; ++c) B.qo[l + c * n] = B.qa[l + c * n];
  }
}

// cofactor metrics from the 9 coordinate derivatives in scr (src/mo_grid.f90:107-115);
// scr field 3*(m-1)+(d-1) = d(coordinate m)/d(xi_d)
__global__ void k_cofactors(const BlockDev* __restrict__ bd) {
  FOR_POINTS(bd[blockIdx.y]) {
    const long long n = B.npad;
    const double* g = B.scr;
    const double q1 = g[l], q2 = g[l + n], q3 = g[l + 2 * n];
    const double a1 = g[l + 3 * n], a2 = g[l + 4 * n], a3 = g[l + 5 * n];
    const double d1 = g[l + 6 * n], d2 = g[l + 7 * n], d3 = g[l + 8 * n];
    B.xim[l] = a2 * d3 - d2 * a3;
    B.xim[l + n] = d2 * q3 - q2 * d3;
    B.xim[l + 2 * n] = q2 * a3 - a2 * q3;
    B.etm[l] = a3 * d1 - d3 * a1;
    B.etm[l + n] = d3 * q1 - q3 * d1;
    B.etm[l + 2 * n] = q3 * a1 - a3 * q1;
    B.zem[l] = a1 * d2 - d1 * a2;
    B.zem[l + n] = d1 * q2 - q1 * d2;
    B.zem[l + 2 * n] = q1 * a2 - a1 * q2;
  }
}

// Jacobian (src/mo_grid.f90:157-159)
__global__ void k_jacobian(const BlockDev* __restrict__ bd) {
  FOR_POINTS(bd[blockIdx.y]) {
    const long long n = B.npad;
    const double* g = B.scr;
    const double *xi = B.xim, *et = B.etm, *ze = B.zem;
    double s = g[l] * xi[l];
    s = s + g[l + n] * et[l];
    s = s + g[l + 2 * n] * ze[l];
    s = s + g[l + 3 * n] * xi[l + n];
    s = s + g[l + 4 * n] * et[l + n];
    s = s + g[l + 5 * n] * ze[l + n];
    s = s + g[l + 6 * n] * xi[l + 2 * n];
    s = s + g[l + 7 * n] * et[l + 2 * n];
    s = s + g[l + 8 * n] * ze[l + 2 * n];
    B.yaco[l] = 3.0 / s;
  }
}

// unit face normals cm{1,2,3} (src/mo_grid.f90:161-186); one thread per face line.
struct CmTask { int b, nn, side, nbs, nj, N, line0; double* cm; };
__global__ void k_face_normals(const BlockDev* __restrict__ bd, const CmTask* __restrict__ tasks,
                               const int* __restrict__ line0s, int ntasks, int nlines) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nlines; g += gridDim.x * blockDim.x) {
    const CmTask& T = tasks[find_task(line0s, ntasks, g)];
    const BlockDev& B = bd[T.b];
    const int jk = g - T.line0, j = jk % T.nj, k = jk / T.nj;
    int x, y, z;
    line_xyz(T.nn, T.side * T.N, j, k, x, y, z);
    const long long l = ((long long)z * B.Y + y) * B.Xp + x;
    const double* met = T.nn == 1 ? B.xim : T.nn == 2 ? B.etm : B.zem;
    const double ya = B.yaco[l];
    const double r0 = ya * met[l], r1 = ya * met[l + B.npad], r2 = ya * met[l + 2 * B.npad];
    const double f = 1.0 / sqrt((r0 * r0 + r1 * r1) + r2 * r2);
    T.cm[jk] = f * r0;
    T.cm[T.nbs + jk] = f * r1;
    T.cm[2 * T.nbs + jk] = f * r2;
  }
}

// junction / surface averaging: snapshot then ordered combination
__global__ void k_avg_snapshot(const BlockDev* __restrict__ bd, const int* __restrict__ sb,
                               const long long* __restrict__ sl, int nsrc, double* __restrict__ snap) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nsrc; e += gridDim.x * blockDim.x) {
    const BlockDev& B = bd[sb[e]];
    const long long l = sl[e];
    for (int c = 0; c < 5; ++c) snap[(long long)e * 5 + c] = B.qa[l + c * B.npad];
  }
}
// mode 0: sum and scale (average_point / average_line); mode 1: running
// average of average_surface.
__global__ void k_avg_combine(const BlockDev* __restrict__ bd, const int* __restrict__ tb,
                              const long long* __restrict__ tl, const int* __restrict__ tfirst,
                              const int* __restrict__ tcount, int ntg, const double* __restrict__ snap, int mode) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntg; t += gridDim.x * blockDim.x) {
    const BlockDev& B = bd[tb[t]];
    const long long l = tl[t];
    const int f = tfirst[t], cnt = tcount[t];
    // all five components formed before any is stored (the stores cannot
    // alias the snapshot, but the compiler cannot know that)
    double out[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      if (mode == 0) {
        double acc = snap[(long long)f * 5 + c];
        for (int j = 1; j < cnt; ++j) acc = acc + snap[(long long)(f + j) * 5 + c];
        out[c] = (1.0 / (double)cnt) * acc;
      } else {
        double q = B.qa[l + c * B.npad];
        double r1 = 1.0;
        for (int j = 0; j < cnt; ++j) {
          r1 = r1 + 1.0;
          const double r2 = 1.0 / r1;
          q = r2 * ((r1 - 1.0) * q + snap[(long long)(f + j) * 5 + c]) + 0.0 * q;
        }
        out[c] = q;
      }
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) B.qa[l + c * B.npad] = out[c];
  }
}

// FP32 copies of the metrics and the Jacobian for the mixed-precision flux path
__global__ void k_metrics_to_f32(const BlockDev* __restrict__ bd) {
  FOR_POINTS(bd[blockIdx.y]) {
    const long long n = B.npad;
    float* xi = const_cast<float*>(B.f.xim);
    float* et = const_cast<float*>(B.f.etm);
    float* ze = const_cast<float*>(B.f.zem);
    for (int c = 0; c < 3; ++c) {
      xi[l + c * n] = float(B.xim[l + c * n]);
      et[l + c * n] = float(B.etm[l + c * n]);
      ze[l + c * n] = float(B.zem[l + c * n]);
    }
    const_cast<float*>(B.f.yaco)[l] = float(B.yaco[l]);
  }
}

// rows of `width` elements between two pitches (host-copy staging <-> padded fields)
__global__ void k_rows_repack(const double* __restrict__ src, int spitch, double* __restrict__ dst, int dpitch,
                              int width, long long rows) {
  const long long n = rows * width;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / width;
    const int x = (int)(e - r * width);
    dst[r * dpitch + x] = src[r * spitch + x];
  }
}

// conversions between an FP64 and an FP32 field of n elements (unit calls)
__global__ void k_f64_to_f32(const double* __restrict__ a, float* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = float(a[i]);
}
__global__ void k_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = double(a[i]);
}

// ---------------------------------------------------------------------------
// Time-step control on the device.

// dt of the step (src/mo_canard_driver.f90:278-294): a new dte from the maxima
// of k_dtmax every tenth step, then the sin^2 ramp from dts to dte. The ramp
// factors sin(0.05 pi k)^2 come from a host table (the same libm values the
// CPU code uses); k past the table falls back to the device sine. Also flags
// the reference's overflow stop (dt == 0 after step 2) seen at step start.
__global__ void k_time_dt(TimeDev* __restrict__ td, const unsigned long long* __restrict__ dtm,
                          const CaseConst* __restrict__ cc, const double* __restrict__ sn2, int nsn2, int ncases,
                          int* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncases) return;
  TimeDev t = td[i];
  if (t.dt == 0.0 && t.n > 2) atomicExch(err, kErrOverflow);
  if (t.n % 10 == 1) {
    t.ndt = t.n;
    t.dts = t.dte;
    const double r1 = __longlong_as_double((long long)dtm[2 * i]);
    const double r2 = __longlong_as_double((long long)dtm[2 * i + 1]);
    const double ra0 = cc[i].cfl / r1;
    double ra1 = ra0;
    if (cc[i].viscous) ra1 = 0.5 / r2;
    t.dte = (ra1 < ra0) ? ra1 : ra0;
  }
  const long long k = t.n - t.ndt;
  double s2;
  if (k >= 0 && k < nsn2) {
    s2 = sn2[k];
  } else {
    const double sn = sin((0.05 * 3.141592653589793) * (double)k);
    s2 = sn * sn;
  }
  t.dt = t.dts + (t.dte - t.dts) * s2;
  td[i] = t;
}

// moving frame (src/mo_physics.f90:144-169); with nsmf = 1 (or a frame at
// rest) it is exact, with the timf ramp it uses the device sine and cosine
__device__ __forceinline__ void movef_dev(const CaseConst& C, double timo, double dtko, double dtk, double umf[3],
                                          double dudtmf[3]) {
  if (C.nsmf == 0) {
    const double pi = 3.141592653589793;
    const double ra0 = pi / C.timf;
    const double ra1 = ra0 * (C.timf < timo ? C.timf : timo);
    const double t2 = timo + dtko;
    const double ra2 = ra0 * (C.timf < t2 ? C.timf : t2);
    double fctr = 1.0 - cos(ra1);
    double dfdt = ra0 * sin(ra2);
    double progmf = 0.5 * (fctr + dtk * dfdt);
    for (int d = 0; d < 3; ++d) umf[d] = progmf * C.uoo[d];
    fctr = sin(ra1);
    dfdt = ra0 * cos(ra2);
    progmf = (0.5 * ra0) * (fctr + dtk * dfdt);
    for (int d = 0; d < 3; ++d) dudtmf[d] = progmf * C.uoo[d];
  } else {
    for (int d = 0; d < 3; ++d) { umf[d] = C.uoo[d]; dudtmf[d] = 0.0; }
  }
}

// stage scalars of stages nk0..nk1 of every case into out[(nk - nk0) * ncases
// + case] (src/mo_canard_driver.f90:261-263, 323-328)
__global__ void k_stage_params(const TimeDev* __restrict__ td, const CaseConst* __restrict__ cc,
                               StageParams* __restrict__ out, int nk0, int nk1, int ncases) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int nst = nk1 - nk0 + 1;
  if (g >= nst * ncases) return;
  const int i = g % ncases, nk = nk0 + g / ncases;
  const TimeDev t = td[i];
  const CaseConst C = cc[i];
  const int nkrk = 4;
  StageParams p;
  const int c1 = min(max(nk - 2, 0), 1), c2 = min(nk - 1, 1);
  double dtko = (t.dt * c1) / (nkrk - nk + 3);
  double dtk = (t.dt * c2) / (nkrk - nk + 2);
  movef_dev(C, t.timo, dtko, dtk, p.umf, p.dudtmf);
  dtko = (t.dt * c2) / (nkrk - nk + 2);
  dtk = t.dt / (nkrk - nk + 1);
  double dud[3];
  movef_dev(C, t.timo, dtko, dtk, p.umfb, dud);
  p.dtk = dtk;
  p.dt = t.dt;
  out[g] = p;
}

// Time-averaged recording (src/mo_canard_driver.f90:373-378): after each step
// qb = qb + (dt/2)(qo + qa) over the stored points of one block, and dtsum += dt.
__global__ void k_record_acc(double* __restrict__ qb, const double* __restrict__ qo,
                             const double* __restrict__ qa, long long npad, int X, int Xp,
                             const TimeDev* __restrict__ td, int icase) {
  const double fctr = 0.5 * td[icase].dt;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < 5 * npad;
       l += (long long)gridDim.x * blockDim.x)
    if ((int)(l % Xp) < X) qb[l] = qb[l] + fctr * (qo[l] + qa[l]);
}
__global__ void k_record_dtsum(double* dtsum, const TimeDev* __restrict__ td, int ncases) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncases) dtsum[c] = dtsum[c] + td[c].dt;
}

// An output of the recording (src/mo_canard_driver.f90:379-402): the average
// qb / dtsum (qo after the first step), written as FP32 rho, u, v, w (plus the
// frame velocity) and p, variable-major in the reference's point order.
__global__ void k_record_out(const double* __restrict__ qb, const double* __restrict__ qo,
                             float* __restrict__ out, int X, int Y, int Z, int Xp, long long npad,
                             const TimeDev* __restrict__ td, const double* __restrict__ dtsum,
                             const StageParams* __restrict__ sp, int icase) {
  const double gamm1 = 1.4 - 1.0;
  const long long n = td[icase].n;
  const double ra0 = 1.0 / dtsum[icase];
  const double* umf = sp[icase].umfb;
  const long long N = (long long)X * Y * Z;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < npad;
       l += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(l % Xp);
    if (x >= X) continue;
    const long long row = l / Xp;  // z * Y + y
    const long long r = row * X + x;
    double q[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) q[c] = (n == 1) ? qo[l + c * npad] : ra0 * qb[l + c * npad];
    const double rr = 1.0 / q[0];
    out[r] = (float)q[0];
#pragma unroll
    for (int c = 1; c < 4; ++c) out[r + c * N] = (float)(rr * q[c] + umf[c - 1]);
    out[r + 4 * N] = (float)(gamm1 * (q[4] - (0.5 * rr) * ((q[1] * q[1] + q[2] * q[2]) + q[3] * q[3])));
  }
}

// wall_condition_update (src/mo_gcbc.f90:424-459) on the wall-face points of all
// blocks. npex is 0 everywhere in the reference (gcbc_init sets it once and
// nothing changes it), so each reset replaces the value; the expressions keep
// the npex terms so that the arithmetic is the reference's. A point on several
// wall faces gets their resets in the reference's face order (nn = 1..3, side
// 0..1): kinds packed two bits each from the low end, 1 inviscid, 2 viscous.
// The frame velocity is the one after movef of the stage (umfb).
__global__ void k_wall_update(const BlockDev* __restrict__ bd, const StageParams* __restrict__ sp,
                              const int* __restrict__ tb, const long long* __restrict__ tl,
                              const int* __restrict__ tk, int n) {
  const double gam = 1.4, hamhamm1 = (1.0 / gam) * (1.0 / (gam - 1.0));
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const BlockDev& B = bd[tb[t]];
    const long long l = tl[t], L = B.npad;
    double* q = B.qa;
    const double* umf = sp[B.case_id].umfb;
    const double npx = 0.0;
    for (int s = 0; s < 3; ++s) {
      const int kind = (tk[t] >> (2 * s)) & 3;
      if (kind == 0) break;
      if (kind == 1) {
        const double ke = (q[l + L] * q[l + L] + q[l + 2 * L] * q[l + 2 * L]) + q[l + 3 * L] * q[l + 3 * L];
        q[l + 4 * L] = npx * q[l + 4 * L] + (1.0 - npx) * (hamhamm1 * pow(q[l], gam) + (0.5 * ke) / q[l]);
      } else {
        const double fctr = (1.0 - npx) * q[l];
        for (int d = 0; d < 3; ++d) q[l + (d + 1) * L] = npx * q[l + (d + 1) * L] - fctr * umf[d];
        const double ke = (q[l + L] * q[l + L] + q[l + 2 * L] * q[l + 2 * L]) + q[l + 3 * L] * q[l + 3 * L];
        q[l + 4 * L] = npx * q[l + 4 * L] + (1.0 - npx) * (hamhamm1 * q[l] + (0.5 * ke) / q[l]);
      }
    }
  }
}

// Self-test of the bounded waits: one warp waits on an mbarrier that nothing
// arrives at. The wait gives up after kWaitNs and raises the timeout flag, as
// a line kernel does when a copy never lands; no fault, no trap.
__global__ void k_wait_selftest(int* __restrict__ err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_done();
  }
  __syncwarp();
  const bool ok = mbar_wait(&bar, 0);
  if (!ok && threadIdx.x == 0) atomicExch(err, kErrTimeout);
}

// n = n + 1, timo = timo + dt (src/mo_canard_driver.f90:369-370)
__global__ void k_time_advance(TimeDev* __restrict__ td, int ncases) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncases) return;
  td[i].n = td[i].n + 1;
  td[i].timo = td[i].timo + td[i].dt;
}

}  // namespace canard
