// Periodic boundary conditions (3dp/): the far images beyond the first
// layer, the dipole correction and the Ewald summation used to check them.
//
// periodic (3dp/traverse_eager.h:46-93): with the source root's multipole
// Mp at the domain centre and cyc = cycle, for each of images-1 sublevels
//   L_root += sum over the 26 x 27 offsets iX = 3*(ix,iy,iz) + (cx,cy,cz),
//             (ix,iy,iz) != 0, of M2L(Mp at offset iX*cyc)       (702 M2L)
//   Mp     += sum over the 26 offsets (ix,iy,iz) != 0 of M2M(Mp from ...)
//   cyc    *= 3.
// M2L and M2M are linear in the offset harmonics, so each sum is one
// translation with the harmonics summed over the offsets; the sums depend
// only on P, the period and the number of images and are kept between
// evaluations.  FP64 in every precision form; the per-thread partial sums are
// reduced in a fixed order, so the result is deterministic.
//
// Dipole correction (3dp/fmm.cxx:63-75): d = sum q X over all bodies,
// coef = 4 pi / (3 cycle^3); p -= coef |d|^2 / N / q, F -= coef d.
//
// Ewald (3dp/ewald.h): wave part by DFT over all sources and inverse DFT at
// the targets (waves with integer k, 0 < |k| <= ksize, in the half space of
// initWaves), real part with erfc over all sources within the cutoff at the
// nearest image per axis, self term -2/sqrt(pi) q alpha.
#include <cmath>
#include <vector>

#include "fmm.cuh"
#include "harmonics.cuh"
#include "translations.cuh"

namespace fmm {

namespace {

constexpr int PT = 256;  // threads of the periodic CTA

// The harmonic sums of the far images, per sublevel l (period cycle * 3^l):
// H[2l] the irregular harmonics summed over the 702 M2L offsets, H[2l + 1]
// the regular harmonics summed over the 26 M2M offsets (rows of nt).  They
// depend only on P, the period and the number of images, so they are made
// once per parameter set and kept.  One CTA; T threads sum the offsets,
// then the partial sums are reduced in thread order (deterministic).
__global__ void __launch_bounds__(PT) k_periodic_harm(int P, int images, double cycle, int T, double2 *H) {
  extern __shared__ double2 sp[];  // partial[T][nt]
  const int nt = tri(P);
  double2 *part = sp;
  const int tid = threadIdx.x;
  double cyc = cycle;
  for (int level = 0; level < images - 1; level++) {
    // irregular harmonics summed over the 702 M2L offsets
    for (int e = tid; e < T * nt; e += PT) part[e] = make_double2(0, 0);
    __syncthreads();
    if (tid < T) {
      double2 *mine = part + (size_t)tid * nt;
      for (int off = tid; off < 702; off += T) {
        const int outer = off / 27, inner = off % 27;
        const int oc = outer < 13 ? outer : outer + 1;  // skip the centre (ix,iy,iz) = 0
        const int ix = oc / 9 - 1, iy = (oc / 3) % 3 - 1, iz = oc % 3 - 1;
        const int cx = inner / 9 - 1, cy = (inner / 3) % 3 - 1, cz = inner % 3 - 1;
        const Sph g = sph_of(-(ix * 3 + cx) * cyc, -(iy * 3 + cy) * cyc, -(iz * 3 + cz) * cyc);
        for (int m = 0; m < P; m++)
          irregular_column(m, P, g.r, g, [&](int n, double2 z) {
            double2 &d = mine[tri(n) + m];
            d.x += z.x;
            d.y += z.y;
          });
      }
    }
    __syncthreads();
    for (int o = tid; o < nt; o += PT) {
      double2 v = make_double2(0, 0);
      for (int t = 0; t < T; t++) {
        v.x += part[(size_t)t * nt + o].x;
        v.y += part[(size_t)t * nt + o].y;
      }
      H[(size_t)(2 * level) * nt + o] = v;
    }
    __syncthreads();
    // regular harmonics summed over the 26 M2M offsets (parent - child)
    for (int e = tid; e < T * nt; e += PT) part[e] = make_double2(0, 0);
    __syncthreads();
    if (tid < 26 && tid < T) {
      double2 *mine = part + (size_t)tid * nt;
      for (int off = tid; off < 26; off += T) {
        const int oc = off < 13 ? off : off + 1;
        const int ix = oc / 9 - 1, iy = (oc / 3) % 3 - 1, iz = oc % 3 - 1;
        const Sph g = sph_of(-ix * cyc, -iy * cyc, -iz * cyc);
        for (int m = 0; m < P; m++)
          regular_column(m, P, g.r, g, g.e, [&](int n, double2 y, double2) {
            double2 &d = mine[tri(n) + m];
            d.x += y.x;
            d.y += y.y;
          });
      }
    }
    __syncthreads();
    for (int o = tid; o < nt; o += PT) {
      double2 v = make_double2(0, 0);
      for (int t = 0; t < T; t++) {
        v.x += part[(size_t)t * nt + o].x;
        v.y += part[(size_t)t * nt + o].y;
      }
      H[(size_t)(2 * level + 1) * nt + o] = v;
    }
    __syncthreads();
    cyc *= 3;
  }
}

// Per evaluation: the root's multipole through the sublevels with the kept
// harmonic sums -- L_root += M2L(Mp, H[2l]), Mp += M2M(Mp, H[2l + 1]).
__global__ void __launch_bounds__(PT) k_periodic(const double2 *M, double2 *L, int P, int images, const double2 *H) {
  extern __shared__ double2 sp[];  // Mp[nt], Mn[nt]
  const int nt = tri(P);
  double2 *Mp = sp, *Mn = Mp + nt;
  const int tid = threadIdx.x;
  for (int o = tid; o < nt; o += PT) Mp[o] = M[o];  // the root is cell 0
  __syncthreads();
  for (int level = 0; level < images - 1; level++) {
    const double2 *H1 = H + (size_t)(2 * level) * nt, *H2 = H1 + nt;
    for (int o = tid; o < nt; o += PT) {
      const int j = order_of(o), k = o - tri(j);
      const double2 v = m2l_coeff(j, k, P, Mp, H1);
      L[o].x += v.x;
      L[o].y += v.y;
    }
    for (int o = tid; o < nt; o += PT) {
      const int j = order_of(o), k = o - tri(j);
      const double2 v = m2m_coeff(j, k, Mp, H2);
      Mn[o] = make_double2(Mp[o].x + v.x, Mp[o].y + v.y);
    }
    __syncthreads();
    for (int o = tid; o < nt; o += PT) Mp[o] = Mn[o];
    __syncthreads();
  }
}

int periodic_threads(int P) {
  const int nt = tri(P);
  int T = 160 * 1024 / (nt * (int)sizeof(double2)) - 3;
  if (T > 64) T = 64;
  if (T < 1) T = 1;
  return T;
}

// ---- dipole correction
constexpr int DB = 256;

// The root's monopole for the far images of the mixed form: the total
// charge, summed in FP64 in a fixed order (block partial sums, then one block
// over the partials in block order).  The mixed upward pass forms it from
// FP32 products, and the far images' lattice sums multiply a spurious net
// charge by their growing image shells: at 60,000 neutral bodies, P = 10,
// the potentials then drifted from the FP64 form's by 5.9e-7, 7.9e-6 and
// 7.0e-4 with 1, 2 and 4 image layers (forces unaffected: the shift is
// nearly constant).
__global__ void k_charge_partial(const double4 *src, long n, double *part) {
  __shared__ double red[DB];
  double q = 0;
  for (long i = (long)blockIdx.x * DB + threadIdx.x; i < n; i += (long)gridDim.x * DB) q += src[i].w;
  red[threadIdx.x] = q;
  __syncthreads();
  for (int s = DB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_root_monopole(const double *part, int nblk, double2 *M) {
  if (threadIdx.x == 0) {
    double q = 0;
    for (int b = 0; b < nblk; b++) q += part[b];
    M[0] = make_double2(q, 0.0);  // M_0^0 of the root (cell 0): the total charge
  }
}

__global__ void k_dipole_partial(const double4 *src, long n, double *part) {
  __shared__ double red[3][DB];
  double d[3] = {0, 0, 0};
  for (long i = (long)blockIdx.x * DB + threadIdx.x; i < n; i += (long)gridDim.x * DB) {
    const double4 b = src[i];
    d[0] += b.x * b.w;
    d[1] += b.y * b.w;
    d[2] += b.z * b.w;
  }
  for (int q = 0; q < 3; q++) red[q][threadIdx.x] = d[q];
  __syncthreads();
  for (int s = DB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int q = 0; q < 3; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; q++) part[blockIdx.x * 3 + q] = red[q][0];
}

__global__ void k_dipole_apply(const double4 *src, double4 *out, long n, const double *part, int nblk,
                               double cycle) {
  double d[3] = {0, 0, 0};
  for (int b = 0; b < nblk; b++)
    for (int q = 0; q < 3; q++) d[q] += part[b * 3 + q];
  const double coef = 4 * M_PI / (3 * cycle * cycle * cycle);
  const double dn = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double4 o = out[i];
    o.x -= coef * dn / (double)n / src[i].w;
    o.y -= coef * d[0];
    o.z -= coef * d[1];
    o.w -= coef * d[2];
    out[i] = o;
  }
}

// ---- Ewald
constexpr int EB = 256;

// One block per wave: structure factor sum_b q_b (cos th, sin th), th = k.x
// scale, scaled by coef exp(-|K|^2 coef2) / |K|^2 (3dp/ewald.h:22-34, :128-141).
__global__ void k_ewald_dft(const int4 *waves, const double4 *src, long n, double scale, double coef, double coef2,
                            double2 *amp) {
  __shared__ double red[2][EB];
  const int4 k = waves[blockIdx.x];
  double re = 0, im = 0;
  for (long i = threadIdx.x; i < n; i += EB) {
    const double4 b = src[i];
    const double th = k.x * b.x * scale + k.y * b.y * scale + k.z * b.z * scale;
    double s, c;
    sincos(th, &s, &c);
    re += b.w * c;
    im += b.w * s;
  }
  red[0][threadIdx.x] = re;
  red[1][threadIdx.x] = im;
  __syncthreads();
  for (int s = EB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double kx = k.x * scale, ky = k.y * scale, kz = k.z * scale;
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double f = coef * exp(-k2 * coef2) / k2;
    amp[blockIdx.x] = make_double2(red[0][0] * f, red[1][0] * f);
  }
}

// Real-space term of one source at the nearest image per axis, inside the
// cutoff (3dp/ewald.h:82-102 realP2P).
__device__ __forceinline__ void ewald_real_pair(double tx, double ty, double tz, const double4 &b, double c2,
                                                double alpha, double a3, double half, double cycle, double &p,
                                                double &fx, double &fy, double &fz) {
  double dx = tx - b.x, dy = ty - b.y, dz = tz - b.z;
  if (dx < -half) dx += cycle;
  if (dx > half) dx -= cycle;
  if (dy < -half) dy += cycle;
  if (dy > half) dy -= cycle;
  if (dz < -half) dz += cycle;
  if (dz > half) dz -= cycle;
  const double R2 = dx * dx + dy * dy + dz * dz;
  if (0 < R2 && R2 < c2) {
    const double R2s = R2 * alpha * alpha, Rs = sqrt(R2s);
    const double invRs = 1 / Rs, invR2s = invRs * invRs, invR3s = invR2s * invRs;
    const double ec = erfc(Rs);
    const double dtmp = b.w * (M_2_SQRTPI * exp(-R2s) * invR2s + ec * invR3s) * a3;
    p += b.w * ec * invRs * alpha;
    fx -= dx * dtmp;
    fy -= dy * dtmp;
    fz -= dz * dtmp;
  }
}

// Inverse DFT term of one wave at a target (3dp/ewald.h:36-51 idft).
__device__ __forceinline__ void ewald_wave_term(double tx, double ty, double tz, const int4 &k, const double2 &a,
                                                double scale, double &p, double &fx, double &fy, double &fz) {
  const double th = k.x * tx * scale + k.y * ty * scale + k.z * tz * scale;
  double s, c;
  sincos(th, &s, &c);
  const double dtmp = a.x * s - a.y * c;
  p += a.x * c + a.y * s;
  fx -= dtmp * k.x * scale;
  fy -= dtmp * k.y * scale;
  fz -= dtmp * k.z * scale;
}

// One block per target (few targets, many sources): the parts selected by
// `parts` -- real part over all sources (nearest image per axis, 0 < R <
// cutoff), the inverse DFT over all waves, the self term; p and F accumulate
// into the target record.
__global__ void k_ewald_target(const double4 *src, long n, const int4 *waves, const double2 *amp, int nw,
                               double scale, double alpha, double cutoff, double cycle, int parts, double *rec) {
  __shared__ double red[4][EB];
  double *r = rec + 8 * (long)blockIdx.x;
  const double tx = r[0], ty = r[1], tz = r[2], tq = r[3];
  double p = 0, fx = 0, fy = 0, fz = 0;
  const double c2 = cutoff * cutoff, a3 = alpha * alpha * alpha, half = cycle / 2;
  if (parts & EXAFMM_EWALD_REAL)
    for (long i = threadIdx.x; i < n; i += EB) ewald_real_pair(tx, ty, tz, src[i], c2, alpha, a3, half, cycle, p, fx, fy, fz);
  if (parts & EXAFMM_EWALD_WAVE)
    for (int w = threadIdx.x; w < nw; w += EB) ewald_wave_term(tx, ty, tz, waves[w], amp[w], scale, p, fx, fy, fz);
  red[0][threadIdx.x] = p;
  red[1][threadIdx.x] = fx;
  red[2][threadIdx.x] = fy;
  red[3][threadIdx.x] = fz;
  __syncthreads();
  for (int s = EB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int q = 0; q < 4; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    r[4] += red[0][0] - ((parts & EXAFMM_EWALD_SELF) ? M_2_SQRTPI * tq * alpha : 0.0);
    r[5] += red[1][0];
    r[6] += red[2][0];
    r[7] += red[3][0];
  }
}

// One thread per target (many targets): sources and waves pass through
// shared memory in tiles of EB, every thread sums its own target.
__global__ void __launch_bounds__(EB) k_ewald_targets(const double4 *src, long n, const int4 *waves,
                                                      const double2 *amp, int nw, double scale, double alpha,
                                                      double cutoff, double cycle, int parts, double *rec, long nt) {
  __shared__ double4 tile[EB];
  __shared__ int4 wtile[EB];
  __shared__ double2 atile[EB];
  const long t = (long)blockIdx.x * EB + threadIdx.x;
  double tx = 0, ty = 0, tz = 0, tq = 0;
  if (t < nt) {
    const double *r = rec + 8 * t;
    tx = r[0]; ty = r[1]; tz = r[2]; tq = r[3];
  }
  double p = 0, fx = 0, fy = 0, fz = 0;
  const double c2 = cutoff * cutoff, a3 = alpha * alpha * alpha, half = cycle / 2;
  if (parts & EXAFMM_EWALD_REAL)
    for (long b = 0; b < n; b += EB) {
      __syncthreads();
      if (b + threadIdx.x < n) tile[threadIdx.x] = src[b + threadIdx.x];
      __syncthreads();
      const int m = (int)min((long)EB, n - b);
      for (int k = 0; k < m; k++) ewald_real_pair(tx, ty, tz, tile[k], c2, alpha, a3, half, cycle, p, fx, fy, fz);
    }
  if (parts & EXAFMM_EWALD_WAVE)
    for (int w0 = 0; w0 < nw; w0 += EB) {
      __syncthreads();
      if (w0 + (int)threadIdx.x < nw) {
        wtile[threadIdx.x] = waves[w0 + threadIdx.x];
        atile[threadIdx.x] = amp[w0 + threadIdx.x];
      }
      __syncthreads();
      const int m = min(EB, nw - w0);
      for (int k = 0; k < m; k++) ewald_wave_term(tx, ty, tz, wtile[k], atile[k], scale, p, fx, fy, fz);
    }
  if (t < nt) {
    double *r = rec + 8 * t;
    r[4] += p - ((parts & EXAFMM_EWALD_SELF) ? M_2_SQRTPI * tq * alpha : 0.0);
    r[5] += fx;
    r[6] += fy;
    r[7] += fz;
  }
}

}  // namespace

void periodic_set_attributes() {
  cudaFuncSetAttribute(k_periodic_harm, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

void periodic_pass(Handle &h) {
  if (h.prm.dim == 2) return periodic_pass_2d(h);
  if (h.prm.images < 2) return;
  const int P = h.prm.P, nt = tri(P), T = periodic_threads(P), images = h.prm.images;
  const double cycle = h.prm.cycle;
  if (!(h.per_P == P && h.per_images == images && h.per_cycle == cycle)) {
    h.per_harm.need((size_t)2 * (images - 1) * nt * sizeof(double2));
    k_periodic_harm<<<1, PT, (size_t)T * nt * sizeof(double2), h.stream>>>(P, images, cycle, T,
                                                                           h.per_harm.as<double2>());
    h.launches++;
    FMM_LAUNCH();
    h.per_P = P;
    h.per_images = images;
    h.per_cycle = cycle;
  }
  if (h.prm.precision == EXAFMM_MIXED) {  // the root's monopole in FP64 (see k_charge_partial)
    const int nblk = 148;
    h.per_part.need(nblk * sizeof(double));
    k_charge_partial<<<nblk, DB, 0, h.stream>>>(h.src.as<double4>(), h.n, h.per_part.as<double>());
    k_root_monopole<<<1, 32, 0, h.stream>>>(h.per_part.as<double>(), nblk, h.M.as<double2>());
    h.launches += 2;
  }
  k_periodic<<<1, PT, (size_t)2 * nt * sizeof(double2), h.stream>>>(h.M.as<double2>(), h.L.as<double2>(), P, images,
                                                                    h.per_harm.as<double2>());
  h.launches++;
  FMM_LAUNCH();
}

void dipole_correction(Handle &h) {
  const int nblk = 148;
  Buf part;
  part.need(nblk * 3 * sizeof(double));
  k_dipole_partial<<<nblk, DB, 0, h.stream>>>(h.src.as<double4>(), h.n, part.as<double>());
  k_dipole_apply<<<grid_for(h.n, 256) < 4096 ? grid_for(h.n, 256) : 4096, 256, 0, h.stream>>>(
      h.src.as<double4>(), h.out.as<double4>(), h.n, part.as<double>(), nblk, h.prm.cycle);
  h.launches += 2;
  FMM_LAUNCH();
  FMM_CUDA(cudaStreamSynchronize(h.stream));
  part.release();
}

void ewald(Handle &h, int parts, int ksize, double alpha, double sigma, double cutoff, double cycle, double *rec_dev,
           long nt) {
  // waves of initWaves (3dp/ewald.h:53-80)
  std::vector<int4> w;
  for (int l = 0; l <= ksize; l++) {
    const int mmin = l == 0 ? 0 : -ksize;
    for (int m = mmin; m <= ksize; m++) {
      const int nmin = (l == 0 && m == 0) ? 1 : -ksize;
      for (int n = nmin; n <= ksize; n++)
        if (l * l + m * m + n * n <= ksize * ksize) w.push_back(make_int4(l, m, n, 0));
    }
  }
  const int nw = (int)w.size();
  Buf wv, amp;
  wv.need(nw * sizeof(int4));
  amp.need(nw * sizeof(double2));
  FMM_CUDA(cudaMemcpyAsync(wv.p, w.data(), nw * sizeof(int4), cudaMemcpyHostToDevice, h.stream));
  const double scale = 2 * M_PI / cycle;
  const double coef = 2 / sigma / cycle / cycle / cycle, coef2 = 1 / (4 * alpha * alpha);
  if (parts & EXAFMM_EWALD_WAVE) {
    k_ewald_dft<<<nw, EB, 0, h.stream>>>(wv.as<int4>(), h.src.as<double4>(), h.n, scale, coef, coef2,
                                         amp.as<double2>());
    h.launches++;
  }
  const long n = (parts & (EXAFMM_EWALD_REAL | EXAFMM_EWALD_WAVE)) ? h.n : 0;
  // a block per target while the targets cannot fill the GPU as threads
  if (nt < 148L * 4 * EB)
    k_ewald_target<<<(unsigned)nt, EB, 0, h.stream>>>(h.src.as<double4>(), n, wv.as<int4>(), amp.as<double2>(), nw,
                                                      scale, alpha, cutoff, cycle, parts, rec_dev);
  else
    k_ewald_targets<<<grid_for(nt, EB), EB, 0, h.stream>>>(h.src.as<double4>(), n, wv.as<int4>(), amp.as<double2>(),
                                                           nw, scale, alpha, cutoff, cycle, parts, rec_dev, nt);
  h.launches++;
  FMM_LAUNCH();
  FMM_CUDA(cudaStreamSynchronize(h.stream));
  wv.release();
  amp.release();
}

}  // namespace fmm
