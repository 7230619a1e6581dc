// tpcf_oracle.cpp -- CPU oracle for the 2pcf pair-summing path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls this
// file; only tests/, the smoke check and the CPU-baseline leg of bench.py load
// it, as the checker.
//
// PARITY STATUS: unpinned.  The reference (tilmantroester/2pcf) is Fortran 90
// and no Fortran compiler exists on this machine or the GPU machines, and the
// reference's own tests hold no golden vector for the pair sums.  The only
// behaviour its tests pin -- kd-tree radius search equals a brute-force scan as
// index sets (src/test_kdtree.f90:96-104) -- is re-checked against this
// restatement by tests/test_oracle.py.
//
// Contents
//   1. ref::  a line-by-line restatement of the reference algorithm, templated
//      on the Fortran `real` kind (float = default build, double = a build with
//      -fdefault-real-8):
//        create_bins / find_bin_index   src/utils.f90:139-230, :101-137
//        grow_tree / search_within_r    src/kdtree.f90:73-205, :207-375
//        tangential_shear_tpcf          src/tpcf.f90:190-378
//        scalar_kappa_tpcf              src/tpcf.f90:380-545
//        partition_data (k-means)       src/kmeans.f90:12-263
//        qsort_arg                      src/utils.f90:239-296
//        covariance_matrix              src/utils.f90:745-764
//   2. canon:: an FP64 brute-force pair sum using the canonical bin rule that
//      the CUDA library also uses (squared FP64 edges, d^2 computed in FP64
//      without contraction), with deterministic summation order.
//   3. det:: the deterministic k-means (fixed-point centroid sums) and the
//      block bootstrap from patch sums, as the CUDA library defines them.
//
// Built with -ffp-contract=off so every float/double expression rounds exactly
// as written.

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#include <omp.h>

namespace {

enum { LIN = 0, LOG = 1, IHS = 2, SQRT = 3 };  // src/utils.f90:7

// Wall times of the last reference pair call: kd-tree build, OpenMP pair loop.
double g_tree_s = 0.0, g_loop_s = 0.0;

// ===================================================================== ref ==
namespace ref {

// Fortran `real` intrinsic helpers for float and double kinds.
inline float  f_log10(float x)  { return log10f(x); }
inline double f_log10(double x) { return log10(x); }
inline float  f_log(float x)    { return logf(x); }
inline double f_log(double x)   { return log(x); }
inline float  f_sqrt(float x)   { return sqrtf(x); }
inline double f_sqrt(double x)  { return sqrt(x); }
inline float  f_pow(float a, float b)   { return powf(a, b); }
inline double f_pow(double a, double b) { return pow(a, b); }
inline float  f_sinh(float x)   { return sinhf(x); }
inline double f_sinh(double x)  { return sinh(x); }
inline float  f_mod(float a, float p)   { return fmodf(a, p); }
inline double f_mod(double a, double p) { return fmod(a, p); }

template <class R> R isinh_transform(R x, R p) {  // src/utils.f90:83-90
  return f_log(p * x + f_sqrt((p * x) * (p * x) + R(1))) / p;
}
template <class R> R sinh_transform(R y, R p) {  // src/utils.f90:92-99
  return f_sinh(p * y) / p;
}

template <class R> struct Binning {  // src/utils.f90:18-24
  R x_min, x_max, bin_size;
  int n_bin, spacing;
  R ihs_theta;
  std::vector<R> edges, centers;
};

// create_bins with (x_min, x_max, n_bin) given -- the only form main.f90:433
// uses.  src/utils.f90:139-230.
template <class R> int create_bins(R x_min, R x_max, int n_bin, int spacing, R p, Binning<R>& b) {
  if (spacing < LIN || spacing > SQRT || n_bin < 1) return 1;
  b.spacing = spacing;
  b.n_bin = n_bin;
  R theta = R(1);
  if (spacing == IHS) { theta = p; }
  b.ihs_theta = theta;
  b.x_min = x_min;
  b.x_max = x_max;
  if (spacing == LIN) b.bin_size = (x_max - x_min) / R(n_bin);
  else if (spacing == LOG) b.bin_size = (f_log10(x_max) - f_log10(x_min)) / R(n_bin);
  else if (spacing == IHS) b.bin_size = (isinh_transform(x_max, theta) - isinh_transform(x_min, theta)) / R(n_bin);
  else b.bin_size = (f_sqrt(x_max) - f_sqrt(x_min)) / R(n_bin);
  b.edges.assign(n_bin + 1, R(0));
  b.centers.assign(n_bin, R(0));
  b.edges[n_bin] = b.x_max;
  for (int i = 1; i <= n_bin; ++i) {
    R e;
    if (spacing == LIN) e = b.x_min + b.bin_size * R(i - 1);
    else if (spacing == LOG) e = f_pow(R(10), f_log10(b.x_min) + b.bin_size * R(i - 1));
    else if (spacing == IHS) e = sinh_transform(isinh_transform(b.x_min, theta) + b.bin_size * R(i - 1), theta);
    else { R s = f_sqrt(b.x_min) + b.bin_size * R(i - 1); e = s * s; }
    b.edges[i - 1] = e;
  }
  for (int i = 0; i < n_bin; ++i) b.centers[i] = b.edges[i] + (b.edges[i + 1] - b.edges[i]) / R(2);
  return 0;
}

// Returns the 0-based bin, or -1.  src/utils.f90:101-137 (1-based there).
template <class R> int find_bin_index(R x, const Binning<R>& b) {
  if (x < b.x_min || x > b.x_max) return -1;
  if (x == b.x_max) return b.n_bin - 1;
  long i;
  if (b.spacing == LIN) {
    i = (long)((x - b.x_min) / b.bin_size) + 1;
  } else if (b.spacing == LOG) {
    R xt = f_log10(x), xm = f_log10(b.x_min);
    i = (long)((xt - xm) / b.bin_size) + 1;
  } else if (b.spacing == IHS) {
    R xt = isinh_transform(x, b.ihs_theta), xm = isinh_transform(b.x_min, b.ihs_theta);
    i = (long)((xt - xm) / b.bin_size) + 1;
  } else {
    R xt = f_sqrt(x), xm = f_sqrt(b.x_min);
    i = (long)((xt - xm) / b.bin_size) + 1;
  }
  if (i > b.n_bin) return -1;  // "Something went wrong during binning."
  return (int)(i - 1);
}

// ---------------------------------------------------------------- kd-tree --
// src/kdtree.f90:10-31 (tree_node, kdtree); indices are 0-based here.
template <class R> struct KDNode {
  int split_dim;
  long l_idx, u_idx;   // 1-based like the reference; 0/0 marks an empty node
  R split_value;
  R bbox[2][2];        // bbox[dim][0=min,1=max]
  KDNode* left;
  KDNode* right;
};

template <class R> struct KDTree {
  long n = 0;
  int leafsize = 10;
  long max_nodes = 0, n_nodes = 0;
  const R* px = nullptr;
  const R* py = nullptr;
  std::vector<long> ind;  // 1-based point indices, as tree%indicies
  std::vector<KDNode<R>*> pool;
  KDNode<R>* root = nullptr;
  bool overflow = false;
  ~KDTree() { for (auto* p : pool) delete p; }
  R coord(long idx1, int d) const { return d == 0 ? px[idx1 - 1] : py[idx1 - 1]; }

  // grow_tree, src/kdtree.f90:73-101
  int grow(const R* x, const R* y, long n_, int leaf) {
    n = n_; px = x; py = y; leafsize = leaf;
    max_nodes = (long)((R)n * f_log((R)n));  // int(n*log(real(n)))
    ind.resize(n);
    for (long i = 0; i < n; ++i) ind[i] = i + 1;
    R bb[2][2];
    bb[0][0] = bb[0][1] = x[0];
    bb[1][0] = bb[1][1] = y[0];
    for (long i = 1; i < n; ++i) {
      bb[0][0] = std::min(bb[0][0], x[i]); bb[0][1] = std::max(bb[0][1], x[i]);
      bb[1][0] = std::min(bb[1][0], y[i]); bb[1][1] = std::max(bb[1][1], y[i]);
    }
    root = build(1, n, bb);
    return overflow ? 1 : 0;
  }

  // build_tree_from_index_range, src/kdtree.f90:103-204
  KDNode<R>* build(long l, long u, const R bbox[2][2]) {
    ++n_nodes;
    KDNode<R>* node = new KDNode<R>();
    pool.push_back(node);
    node->left = node->right = nullptr;
    std::memcpy(node->bbox, bbox, sizeof(node->bbox));
    node->l_idx = l; node->u_idx = u;
    node->split_dim = 0; node->split_value = 0;
    if (n_nodes > max_nodes) {  // "Reached maximum number of nodes ... Aborting."
      overflow = true;
      node->l_idx = node->u_idx = 0;
      return node;
    }
    if (u - l + 1 <= leafsize) {
      if (u - l + 1 > 0) {
        for (int d = 0; d < 2; ++d) {
          R mn = coord(ind[l - 1], d), mx = mn;
          for (long i = l; i <= u; ++i) { R v = coord(ind[i - 1], d); mn = std::min(mn, v); mx = std::max(mx, v); }
          node->bbox[d][0] = mn; node->bbox[d][1] = mx;
        }
      } else {
        node->l_idx = 0; node->u_idx = 0;
      }
      return node;
    }
    // maxloc(bbox(:,2) - bbox(:,1)): first maximum
    int sd = ((bbox[1][1] - bbox[1][0]) > (bbox[0][1] - bbox[0][0])) ? 1 : 0;
    node->split_dim = sd;
    R mid = (bbox[sd][0] + bbox[sd][1]) / R(2);
    long lt = l, ut = u;
    while (lt < ut) {
      if (coord(ind[lt - 1], sd) <= mid) {
        ++lt;
      } else {
        std::swap(ind[lt - 1], ind[ut - 1]);
        --ut;
      }
    }
    if (coord(ind[lt - 1], sd) > mid) --lt;
    node->split_value = mid;
    R lb[2][2], rb[2][2];
    std::memcpy(lb, bbox, sizeof(lb));
    std::memcpy(rb, bbox, sizeof(rb));
    lb[sd][1] = mid;
    rb[sd][0] = mid;
    if (l > lt) std::memcpy(lb, rb, sizeof(lb));
    else if (lt + 1 > u) std::memcpy(rb, lb, sizeof(rb));
    node->left = build(l, lt, lb);
    if (overflow) return node;
    node->right = build(lt + 1, u, rb);
    if (overflow) return node;
    for (int d = 0; d < 2; ++d) {
      node->bbox[d][0] = std::min(node->left->bbox[d][0], node->right->bbox[d][0]);
      node->bbox[d][1] = std::max(node->left->bbox[d][1], node->right->bbox[d][1]);
    }
    return node;
  }

  // max_distance_to_box, src/kdtree.f90:323-345
  R max_dist(const R bb[2][2], R qx, R qy) const {
    R q[2] = {qx, qy}, dist = 0;
    for (int i = 0; i < 2; ++i) {
      R dl = (bb[i][0] - q[i]) * (bb[i][0] - q[i]);
      R dr = (bb[i][1] - q[i]) * (bb[i][1] - q[i]);
      dist = dist + (dl > dr ? dl : dr);
    }
    return f_sqrt(dist);
  }
  // min_distance_to_box, src/kdtree.f90:347-374
  R min_dist(const R bb[2][2], R qx, R qy) const {
    R q[2] = {qx, qy}, dist = 0;
    for (int i = 0; i < 2; ++i) {
      R dl = bb[i][0] - q[i], dr = bb[i][1] - q[i];
      R dl2 = dl * dl, dr2 = dr * dr;
      if (dl < R(0) && dr > R(0)) continue;
      dist = dist + (dl2 > dr2 ? dr2 : dl2);
    }
    return f_sqrt(dist);
  }

  // search_index_range_within_r, src/kdtree.f90:302-321
  void scan(R qx, R qy, R r, long l, long u, long* res, long cap, long& nf, int& err) const {
    for (long i = l; i <= u; ++i) {
      R dx = coord(ind[i - 1], 0) - qx, dy = coord(ind[i - 1], 1) - qy;
      if (dx * dx + dy * dy <= r * r) {
        ++nf;
        if (nf > cap) { err = 2; return; }  // reference prints and returns
        res[nf - 1] = ind[i - 1];
      }
    }
  }

  // search_node_within_r, src/kdtree.f90:234-300
  void search_node(const KDNode<R>* node, R qx, R qy, R r, long* res, long cap, long& nf, int& err) const {
    if (node->l_idx == 0) return;
    if (min_dist(node->bbox, qx, qy) > r) return;
    if (max_dist(node->bbox, qx, qy) <= r) {
      if (nf + node->u_idx - node->l_idx + 1 > cap) { err = 1; return; }  // reference: stop
      for (long i = node->l_idx; i <= node->u_idx; ++i) res[nf++] = ind[i - 1];
      return;
    }
    if (!node->left && !node->right) { scan(qx, qy, r, node->l_idx, node->u_idx, res, cap, nf, err); return; }
    R q = node->split_dim == 0 ? qx : qy;
    R dts = q - node->split_value;
    if (dts * dts > r * r) {
      if (dts < R(0)) search_node(node->left, qx, qy, r, res, cap, nf, err);
      else search_node(node->right, qx, qy, r, res, cap, nf, err);
    } else {
      search_node(node->left, qx, qy, r, res, cap, nf, err);
      if (err == 1) return;
      search_node(node->right, qx, qy, r, res, cap, nf, err);
    }
  }

  // search_within_r, src/kdtree.f90:207-232.  Results are 1-based indices.
  int search(R qx, R qy, R r, long* res, long cap, long& nf, bool brute) const {
    nf = 0;
    int err = 0;
    if (brute) scan(qx, qy, r, root->l_idx, root->u_idx, res, cap, nf, err);
    else search_node(root, qx, qy, r, res, cap, nf, err);
    return err;
  }
};

// ---------------------------------------------------------- pair loops ------
template <class R> struct PairOut {
  R* avg_theta; R* g_t; R* g_x; R* weights; long long* n_pairs;
  R* xi_E; R* xi_B; R* K_m; R* w_m; R* marks_weight;  // nullable
};

// mode 0: tangential_shear_tpcf  (src/tpcf.f90:190-378)
// mode 1: scalar_kappa_tpcf      (src/tpcf.f90:380-545)
// For mode 1 the B arrays are x, y, kappa_E (e1 slot), kappa_B (e2 slot), w;
// zA, zB and mB are ignored.  Returns 0, or 1/2 on kd result-buffer overflow
// (the reference stops or reads past its buffer there), 3 on tree overflow.
template <class R>
int pair_loop(int mode, long nA, const R* xA, const R* yA, const R* zA, const R* valA, const R* wA,
              long nB, const R* xB, const R* yB, const R* zB, const R* e1B, const R* e2B,
              const R* wB, const R* mB, const Binning<R>& bins, bool use_kd_tree, int num_threads,
              PairOut<R> o) {
  const int nb = bins.n_bin;
  R xmn = xB[0], xmx = xB[0], ymn = yB[0], ymx = yB[0];
  for (long i = 1; i < nB; ++i) {
    xmn = std::min(xmn, xB[i]); xmx = std::max(xmx, xB[i]);
    ymn = std::min(ymn, yB[i]); ymx = std::max(ymx, yB[i]);
  }
  R x_range = xmx - xmn, y_range = ymx - ymn;
  R point_density = R(nB) / (x_range * y_range);
  const R pi = R(3.141592653589793);
  // approx_points_in_theta_max_ball = pi*bins%x_max**2 * point_density
  long approx = (long)(pi * (bins.x_max * bins.x_max) * point_density);
  long cap = (long)(R(approx) * R(10.0));

  std::vector<R> avg(nb, 0), gt(nb, 0), gx(nb, 0), wsum(nb, 0), K(nb, 0);
  std::vector<long long> np(nb, 0);
  if (o.xi_E) {
    std::fill(o.xi_E, o.xi_E + (size_t)nb * nA, R(0));
    std::fill(o.xi_B, o.xi_B + (size_t)nb * nA, R(0));
    std::fill(o.K_m, o.K_m + (size_t)nb * nA, R(0));
    std::fill(o.w_m, o.w_m + (size_t)nb * nA, R(0));
    std::fill(o.marks_weight, o.marks_weight + nA, R(0));
  }
  KDTree<R> tree;
  const double t0 = omp_get_wtime();
  if (use_kd_tree) {
    if (tree.grow(xB, yB, nB, 10)) return 3;
  }
  const double t1 = omp_get_wtime();
  int status = 0;
  const R r = bins.x_max;
#pragma omp parallel num_threads(num_threads)
  {
    std::vector<R> lavg(nb, 0), lgt(nb, 0), lgx(nb, 0), lw(nb, 0), lK(nb, 0);
    std::vector<long long> lnp(nb, 0);
    std::vector<long> res(use_kd_tree ? std::max(cap, 1L) : 0);
#pragma omp for schedule(static)
    for (long i = 0; i < nA; ++i) {
      R xf = xA[i], yf = yA[i], vf = valA[i], wf = wA[i];
      R zf = mode == 0 ? zA[i] : R(0);
      if (wf == R(0)) continue;
      long nfound;
      if (use_kd_tree) {
        int e = tree.search(xf, yf, r, res.data(), cap, nfound, false);
        if (e) {
#pragma omp critical
          status = e;
          continue;
        }
      } else {
        nfound = nB;
      }
      for (long jj = 0; jj < nfound; ++jj) {
        long j = use_kd_tree ? res[jj] - 1 : jj;
        if (mode == 0) {
          R zb = zB[j];
          if (zf < R(0) || zb < R(0)) continue;
          R dx = xf - xB[j], dy = yf - yB[j];
          R dist = f_sqrt(dx * dx + dy * dy);
          if (zf > zb) continue;
          int b = find_bin_index(dist, bins);
          if (b < 0) continue;
          R w = wB[j], m = mB[j], e1 = e1B[j], e2 = e2B[j];
          R cos2phi = R(2) * ((dx / dist) * (dx / dist)) - R(1);
          R sin2phi = R(2) * dx * dy / (dist * dist);
          R tt = (e1 * cos2phi + e2 * sin2phi) * w * vf * wf;
          R tx = (-e1 * sin2phi + e2 * cos2phi) * w * vf * wf;
          lavg[b] = lavg[b] + dist * w * wf;
          lgt[b] = lgt[b] - tt;
          lgx[b] = lgx[b] - tx;
          lw[b] = lw[b] + w * wf;
          lnp[b] += 1;
          lK[b] = lK[b] + w * (R(1) + m) * wf;
          if (o.xi_E) {
            size_t k = (size_t)i * nb + b;
            o.xi_E[k] = o.xi_E[k] - tt;
            o.xi_B[k] = o.xi_B[k] - tx;
            o.w_m[k] = o.w_m[k] + w * wf;
            o.K_m[k] = o.K_m[k] + w * (R(1) + m) * wf;
            o.marks_weight[i] = o.marks_weight[i] + w * wf;
          }
        } else {
          R dx = xf - xB[j], dy = yf - yB[j];
          R dist = f_sqrt(dx * dx + dy * dy);
          int b = find_bin_index(dist, bins);
          if (b < 0) continue;
          R w = wB[j], kE = e1B[j], kB = e2B[j];
          R tE = kE * w * vf * wf, tB = kB * w * vf * wf;
          lavg[b] = lavg[b] + dist * w * wf;
          lgt[b] = lgt[b] + tE;
          lgx[b] = lgx[b] + tB;
          lw[b] = lw[b] + w * wf;
          lnp[b] += 1;
          lK[b] = lK[b] + w * wf;
          if (o.xi_E) {
            size_t k = (size_t)i * nb + b;
            o.xi_E[k] = o.xi_E[k] + tE;
            o.xi_B[k] = o.xi_B[k] + tB;
            o.w_m[k] = o.w_m[k] + w * wf;
            o.K_m[k] = o.K_m[k] + w * wf;
            o.marks_weight[i] = o.marks_weight[i] + w * wf;
          }
        }
      }
    }
#pragma omp critical
    {
      for (int b = 0; b < nb; ++b) {
        avg[b] += lavg[b]; gt[b] += lgt[b]; gx[b] += lgx[b];
        wsum[b] += lw[b]; K[b] += lK[b]; np[b] += lnp[b];
      }
    }
  }
  g_tree_s = t1 - t0;
  g_loop_s = omp_get_wtime() - t1;
  // normalisation, src/tpcf.f90:369-376
  for (int b = 0; b < nb; ++b) {
    o.avg_theta[b] = avg[b] / wsum[b];
    if (K[b] > R(0)) { o.g_t[b] = gt[b] / K[b]; o.g_x[b] = gx[b] / K[b]; }
    else { o.g_t[b] = 0; o.g_x[b] = 0; }
    o.weights[b] = wsum[b];
    o.n_pairs[b] = np[b];
  }
  return status;
}

// ----------------------------------------------------- qsort_arg (utils) ----
// src/utils.f90:239-296: Hoare-partition quicksort returning an argsort.
template <class T> void qsort_arg(const T* a, long n, long* order, bool reverse) {
  std::vector<T> w(a, a + n);
  for (long i = 0; i < n; ++i) order[i] = i;
  struct S {
    static void qs(std::vector<T>& w, long* order, long l, long r) {  // 0-based inclusive
      T pivot = w[(l + r + 2) / 2 - 1];
      long i = l - 1, j = r + 1;
      for (;;) {
        do { --j; } while (!(w[j] <= pivot));
        do { ++i; } while (!(w[i] >= pivot));
        if (i < j) {
          std::swap(w[i], w[j]);
          std::swap(order[i], order[j]);
        } else if (i == j) {
          ++i;
          break;
        } else {
          break;
        }
      }
      if (l < j) qs(w, order, l, j);
      if (i < r) qs(w, order, i, r);
    }
  };
  if (n > 1) S::qs(w, order, 0, n - 1);
  if (reverse) std::reverse(order, order + n);
}

// ------------------------------------------------- partition_data (k-means) --
// src/kmeans.f90:12-263 in FP32 (or double), serial (n_threads = 1), with the
// fixed-grid initial centroids (kmeans.f90:85-112).  Labels are 0-based.
template <class R>
int partition_data(long n, const R* x, const R* y, const R* wts, int k, bool equal_size,
                   R scaling, int max_iterations, R reassignment_tolerance, R weight_tolerance,
                   int* labels, R* cx, R* cy, int* n_iter_out) {
  if (k <= 1) return 1;
  std::vector<long> cand_idx(equal_size ? n : 0);
  std::vector<R> cand_memb(equal_size ? n : 0, R(0));
  R mean_cw = 0;
  for (long i = 0; i < n; ++i) mean_cw = mean_cw + wts[i];
  mean_cw = mean_cw / R(k);
  R xmn = x[0], xmx = x[0], ymn = y[0], ymx = y[0];
  for (long i = 1; i < n; ++i) {
    xmn = std::min(xmn, x[i]); xmx = std::max(xmx, x[i]);
    ymn = std::min(ymn, y[i]); ymx = std::max(ymx, y[i]);
  }
  R diam = f_sqrt((xmx - xmn) * (xmx - xmn) + (ymx - ymn) * (ymx - ymn));
  int n_side = (int)f_sqrt(R(k));
  if (xmx - xmn > ymx - ymn) {
    R dy = (ymx - ymn) / R(n_side);
    R dx = (xmx - xmn) * R(n_side) / R(k);
    for (int j = 1; j <= k; ++j) {
      int row = (int)((dx / R(2) + dx * R(j - 1)) / (xmx - xmn));
      cx[j - 1] = xmn + f_mod(dx / R(2) + dx * R(j - 1), xmx - xmn);
      cy[j - 1] = ymn + dy / R(2) + dy * R(row);
    }
  } else {
    R dx = (xmx - xmn) / R(n_side);
    R dy = (ymx - ymn) * R(n_side) / R(k);
    for (int j = 1; j <= k; ++j) {
      int row = (int)((dy / R(2) + dy * R(j - 1)) / (ymx - ymn));
      cy[j - 1] = ymn + f_mod(dy / R(2) + dy * R(j - 1), ymx - ymn);
      cx[j - 1] = xmn + dx / R(2) + dx * R(row);
    }
  }
  // cluster_indicies = real(i-1)/n_data*k + 1   (1-based), stored 1-based here
  std::vector<int> lab(n);
  for (long i = 0; i < n; ++i) lab[i] = (int)(R(i) / R(n) * R(k) + R(1));
  std::vector<R> cw(k + 1, R(0));
  for (int j = 1; j <= k; ++j) {
    R s = 0;
    for (long i = 0; i < n; ++i) if (lab[i] == j) s = s + wts[i];
    cw[j] = s;
  }
  int n_iter = 0;
  long n_re = 0;
  R max_dev = 0;
  while (n_iter <= max_iterations) {
    ++n_iter;
    n_re = 0;
    // assign_clusters, src/kmeans.f90:162-208 (serial order)
    for (long i = 0; i < n; ++i) {
      R min_d = diam * R(10);
      int ci = 0;
      for (int j = 1; j <= k; ++j) {
        R dw = (n_iter > 1 && scaling > R(0)) ? R(1) + (cw[j] / mean_cw - R(1)) * scaling : R(1);
        R ddx = x[i] - cx[j - 1], ddy = y[i] - cy[j - 1];
        R d = dw * f_sqrt(ddx * ddx + ddy * ddy);
        if (equal_size && n_iter > 1 && d > R(0)) {
          if (d < min_d) {
            cand_memb[i] = min_d / d;
            cand_idx[i] = ci;
            min_d = d;
            ci = j;
          } else if (d < cand_memb[i] * min_d) {
            cand_memb[i] = d / min_d;
            cand_idx[i] = j;
          }
        } else if (d < min_d) {
          min_d = d;
          ci = j;
        }
      }
      if (ci != lab[i]) {
        int old = lab[i];
        lab[i] = ci;
        cw[old] = cw[old] - wts[i];
        cw[ci] = cw[ci] + wts[i];
        ++n_re;
      }
    }
    // calculate_centroids, src/kmeans.f90:210-219
    std::vector<R> sx(k + 1, R(0)), sy(k + 1, R(0));
    for (long i = 0; i < n; ++i) {
      sx[lab[i]] = sx[lab[i]] + x[i] * wts[i];
      sy[lab[i]] = sy[lab[i]] + y[i] * wts[i];
    }
    for (int j = 1; j <= k; ++j) { cx[j - 1] = sx[j] / cw[j]; cy[j - 1] = sy[j] / cw[j]; }
    R mx = cw[1], mn = cw[1];
    for (int j = 2; j <= k; ++j) { mx = std::max(mx, cw[j]); mn = std::min(mn, cw[j]); }
    max_dev = (mx - mn) / mean_cw;
    if (n_re == 0) break;
    if (R(n_re) / R(n) < reassignment_tolerance) break;
  }
  // postprocess_weights, src/kmeans.f90:221-262
  if (equal_size && max_dev > weight_tolerance) {
    std::vector<long> size_order(k), cand_order(n);
    qsort_arg(cw.data() + 1, k, size_order.data(), true);
    qsort_arg(cand_memb.data(), n, cand_order.data(), false);
    for (int jj = 0; jj < k; ++jj) {
      int c = (int)size_order[jj] + 1;
      std::vector<long> members, transfer;
      for (long t = 0; t < n; ++t) {
        long di = cand_order[t];
        if (lab[di] == c) { members.push_back(di); transfer.push_back(cand_idx[di]); }
      }
      for (size_t t = 0; t < members.size(); ++t) {
        long di = members[t];
        long dest = transfer[t];
        if (dest == 0) continue;
        bool heavier = false;
        for (int q = 0; q <= jj; ++q) if (size_order[q] + 1 == dest) heavier = true;
        if (heavier) continue;
        lab[di] = (int)dest;
        cw[c] = cw[c] - wts[di];
        cw[dest] = cw[dest] + wts[di];
        if (cw[c] <= mean_cw * (R(1) + weight_tolerance)) break;
      }
    }
  }
  for (long i = 0; i < n; ++i) labels[i] = lab[i] - 1;
  if (n_iter_out) *n_iter_out = n_iter;
  return 0;
}

}  // namespace ref

// =================================================================== canon ==
namespace canon {

// Canonical FP64 edges.  The CUDA library's host code evaluates the same
// formulas (same libm) and uploads edges^2 to the device.
int edges(double x_min, double x_max, int n_bin, int spacing, double p, double* e, double* e2) {
  if (n_bin < 1 || !(x_max > x_min) || spacing < LIN || spacing > SQRT) return 1;
  if (spacing == LOG && !(x_min > 0)) return 1;
  if (spacing == SQRT && !(x_min >= 0)) return 1;
  if (spacing == IHS && !(p > 0)) return 1;
  e[0] = x_min;
  e[n_bin] = x_max;
  if (spacing == LIN) {
    double d = (x_max - x_min) / n_bin;
    for (int i = 1; i < n_bin; ++i) e[i] = x_min + i * d;
  } else if (spacing == LOG) {
    double l0 = log10(x_min), d = (log10(x_max) - l0) / n_bin;
    for (int i = 1; i < n_bin; ++i) e[i] = pow(10.0, l0 + i * d);
  } else if (spacing == SQRT) {
    double s0 = sqrt(x_min), d = (sqrt(x_max) - s0) / n_bin;
    for (int i = 1; i < n_bin; ++i) { double s = s0 + i * d; e[i] = s * s; }
  } else {
    double t0 = log(p * x_min + sqrt((p * x_min) * (p * x_min) + 1.0)) / p;
    double t1 = log(p * x_max + sqrt((p * x_max) * (p * x_max) + 1.0)) / p;
    double d = (t1 - t0) / n_bin;
    for (int i = 1; i < n_bin; ++i) e[i] = sinh(p * (t0 + i * d)) / p;
  }
  for (int i = 0; i <= n_bin; ++i) e2[i] = e[i] * e[i];
  for (int i = 0; i < n_bin; ++i) if (!(e2[i + 1] > e2[i])) return 1;
  return 0;
}

// Canonical bin of d2 (FP64): -1 outside [e2[0], e2[n]]; n-1 at d2 == e2[n];
// otherwise the largest i < n with e2[i] <= d2.
inline int bin_of(double d2, const double* e2, int n) {
  if (!(d2 >= e2[0]) || d2 > e2[n]) return -1;
  if (d2 == e2[n]) return n - 1;
  int lo = 0, hi = n;  // e2[lo] <= d2 < e2[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (d2 >= e2[mid]) lo = mid; else hi = mid;
  }
  return lo;
}

inline double d2_of(float xa, float ya, float xb, float yb) {
  double dx = (double)xa - (double)xb;
  double dy = (double)ya - (double)yb;
  double a = dx * dx;
  double b = dy * dy;
  return a + b;
}

// Q_AGT/Q_AGX: sums of |g_t term|, |g_x term|.  Q_NGT/Q_NGX: sums of the
// bound on each term's size before the rotation, w_B |val_A w_A| |(e1, e2)|
// for shear (both rows) and |term| for scalar fields: an FP32 evaluation of
// the rotated term errs by a few ulps of that bound, not of the term itself.
enum { Q_DW = 0, Q_GT, Q_GX, Q_W, Q_K, Q_N, Q_AGT, Q_AGX, Q_NGT, Q_NGX, NQ };

// One lens against all sources, FP64, canonical binning.  acc is [NQ][n_bin].
inline void lens_row(int mode, float xa, float ya, float za, float va, float wa,
                     long nB, const float* xB, const float* yB, const float* zB,
                     const float* e1B, const float* e2B, const float* wB, const float* mB,
                     const double* e2, int nb, double* acc) {
  const double e2max = e2[nb];
  if (wa == 0.0f) return;
  if (mode == 0 && za < 0.0f) return;
  for (long j = 0; j < nB; ++j) {
    if (mode == 0) {
      float zb = zB[j];
      if (zb < 0.0f || za > zb) continue;
    }
    double d2 = d2_of(xa, ya, xB[j], yB[j]);
    if (d2 > e2max) continue;
    int b = bin_of(d2, e2, nb);
    if (b < 0) continue;
    double dx = (double)xa - (double)xB[j];
    double dy = (double)ya - (double)yB[j];
    double d = sqrt(d2);
    double w = (double)wB[j], vw = (double)va * (double)wa;
    double tt, tx, kk;
    if (mode == 0) {
      double c2 = 2.0 * ((dx / d) * (dx / d)) - 1.0;
      double s2 = 2.0 * dx * dy / d2;
      double e1 = e1B[j], ee2 = e2B[j];
      tt = -(e1 * c2 + ee2 * s2) * w * vw;
      tx = -(-e1 * s2 + ee2 * c2) * w * vw;
      kk = w * (1.0 + (double)mB[j]) * (double)wa;
    } else {
      tt = (double)e1B[j] * w * vw;
      tx = (double)e2B[j] * w * vw;
      kk = w * (double)wa;
    }
    double* a = acc;
    a[Q_DW * nb + b] += d * w * (double)wa;
    a[Q_GT * nb + b] += tt;
    a[Q_GX * nb + b] += tx;
    a[Q_W * nb + b] += w * (double)wa;
    a[Q_K * nb + b] += kk;
    a[Q_N * nb + b] += 1.0;
    a[Q_AGT * nb + b] += fabs(tt);
    a[Q_AGX * nb + b] += fabs(tx);
    const double nt = mode == 0 ? hypot((double)e1B[j], (double)e2B[j]) * w * fabs(vw) : fabs(tt);
    a[Q_NGT * nb + b] += nt;
    a[Q_NGX * nb + b] += mode == 0 ? nt : fabs(tx);
  }
}

}  // namespace canon

// ===================================================================== det ==
namespace det {

// Fixed-point scale rule shared with the CUDA library: the largest s such that
// n * max|v| * 2^s < 2^62, clamped to [0, 60].
inline int fixed_scale(long n, double vmax) {
  if (!(vmax > 0)) return 60;
  int e;
  frexp((double)n * vmax, &e);  // n*vmax < 2^e
  int s = 62 - e;
  return std::max(0, std::min(60, s));
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the counter-based RNG the
// library's bootstrap kernel uses.  Host replica.
inline void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Draw d of sample s: counter (d/4, s, 0x2pcf, 0), key = seed; the 32-bit word
// d%4 mapped to [0, n) by multiply-shift.
inline uint32_t draw(uint64_t seed, uint32_t s, uint32_t d, uint32_t n) {
  uint32_t c[4] = {d >> 2, s, 0x2BCFu, 0u};
  philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  uint32_t r = c[d & 3];
  return (uint32_t)(((uint64_t)r * n) >> 32);
}

}  // namespace det

}  // namespace

// ================================================================ C exports ==
extern "C" {

int orc_version() { return 1; }

void orc_last_timing(double* tree_s, double* loop_s) {
  *tree_s = g_tree_s;
  *loop_s = g_loop_s;
}

int orc_create_bins_f32(float x_min, float x_max, int n_bin, int spacing, float p,
                        float* edges, float* centers, float* bin_size) {
  ref::Binning<float> b;
  if (ref::create_bins<float>(x_min, x_max, n_bin, spacing, p, b)) return 1;
  std::copy(b.edges.begin(), b.edges.end(), edges);
  std::copy(b.centers.begin(), b.centers.end(), centers);
  *bin_size = b.bin_size;
  return 0;
}

int orc_find_bin_f32(const float* d, long n, float x_min, float x_max, int n_bin, int spacing,
                     float p, int* out) {
  ref::Binning<float> b;
  if (ref::create_bins<float>(x_min, x_max, n_bin, spacing, p, b)) return 1;
  for (long i = 0; i < n; ++i) out[i] = ref::find_bin_index(d[i], b);
  return 0;
}

int orc_canonical_edges(double x_min, double x_max, int n_bin, int spacing, double p,
                        double* edges, double* edges_sq) {
  return canon::edges(x_min, x_max, n_bin, spacing, p, edges, edges_sq);
}

int orc_canonical_bin(const double* d2, long n, const double* e2, int n_bin, int* out) {
  for (long i = 0; i < n; ++i) out[i] = canon::bin_of(d2[i], e2, n_bin);
  return 0;
}

#define REF_PAIR_EXPORT(NAME, R)                                                                 \
  int NAME(int mode, long nA, const R* xA, const R* yA, const R* zA, const R* valA, const R* wA, \
           long nB, const R* xB, const R* yB, const R* zB, const R* e1B, const R* e2B,           \
           const R* wB, const R* mB, R x_min, R x_max, int n_bin, int spacing, R p,              \
           int use_kd_tree, int num_threads, R* avg_theta, R* g_t, R* g_x, R* weights,          \
           long long* n_pairs, R* xi_E, R* xi_B, R* K_m, R* w_m, R* marks_weight) {              \
    ref::Binning<R> b;                                                                           \
    if (ref::create_bins<R>(x_min, x_max, n_bin, spacing, p, b)) return 10;                      \
    ref::PairOut<R> o{avg_theta, g_t, g_x, weights, n_pairs, xi_E, xi_B, K_m, w_m, marks_weight}; \
    return ref::pair_loop<R>(mode, nA, xA, yA, zA, valA, wA, nB, xB, yB, zB, e1B, e2B, wB, mB,  \
                             b, use_kd_tree != 0, num_threads, o);                               \
  }
REF_PAIR_EXPORT(orc_ref_pairs_f32, float)
REF_PAIR_EXPORT(orc_ref_pairs_f64, double)

// Canonical FP64 pair sums.
//   sums: [10][n_bin] = (sum d*wA*wB, sum g_t terms, sum g_x terms, sum wA*wB,
//                        sum K terms, n_pairs, sum |g_t terms|, sum |g_x terms|,
//                        the two term-bound rows Q_NGT, Q_NGX)
//   lens_idx/lens_out (optional): per-lens [n_sel][10][n_bin] of the same
//   quantities for the listed lens indices.
// Summation order is fixed (per lens over sources in index order, then lenses
// in blocks of 64 in index order), so results do not depend on num_threads.
int orc_canon_pairs(int mode, long nA, const float* xA, const float* yA, const float* zA,
                    const float* valA, const float* wA, long nB, const float* xB, const float* yB,
                    const float* zB, const float* e1B, const float* e2B, const float* wB,
                    const float* mB, const double* e2, int n_bin, int num_threads, double* sums,
                    const long* lens_idx, long n_sel, double* lens_out) {
  const int nb = n_bin, NQ = canon::NQ;
  std::fill(sums, sums + (size_t)NQ * nb, 0.0);
  if (!lens_idx) {
    const long CH = 64;
    long nch = (nA + CH - 1) / CH;
    std::vector<double> part((size_t)nch * NQ * nb, 0.0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads)
    for (long c = 0; c < nch; ++c) {
      std::vector<double> acc((size_t)NQ * nb);
      double* pc = part.data() + (size_t)c * NQ * nb;
      for (long i = c * CH; i < std::min(nA, (c + 1) * CH); ++i) {
        std::fill(acc.begin(), acc.end(), 0.0);
        canon::lens_row(mode, xA[i], yA[i], mode == 0 ? zA[i] : 0.0f, valA[i], wA[i], nB, xB, yB,
                        zB, e1B, e2B, wB, mB, e2, nb, acc.data());
        for (int q = 0; q < NQ * nb; ++q) pc[q] += acc[q];
      }
    }
    for (long c = 0; c < nch; ++c)
      for (int q = 0; q < NQ * nb; ++q) sums[q] += part[(size_t)c * NQ * nb + q];
  } else {
    std::vector<double> all((size_t)n_sel * NQ * nb, 0.0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads)
    for (long s = 0; s < n_sel; ++s) {
      long i = lens_idx[s];
      double* acc = all.data() + (size_t)s * NQ * nb;
      canon::lens_row(mode, xA[i], yA[i], mode == 0 ? zA[i] : 0.0f, valA[i], wA[i], nB, xB, yB,
                      zB, e1B, e2B, wB, mB, e2, nb, acc);
    }
    for (long s = 0; s < n_sel; ++s) {
      const double* acc = all.data() + (size_t)s * NQ * nb;
      for (int q = 0; q < NQ * nb; ++q) sums[q] += acc[q];
      if (lens_out)  // all NQ rows: d*w, g_t, g_x, w, K, n, sum|g_t terms|, sum|g_x terms|, the two bound rows
        for (int q = 0; q < NQ * nb; ++q) lens_out[(size_t)s * NQ * nb + q] = acc[q];
    }
  }
  return 0;
}

// FP64 brute-force gradient of L = sum_b lt[b]*xi_t,b + lx[b]*xi_x,b of the
// shear-scalar estimator (canonical bins), with respect to val_A, w_A (per
// lens) and e1_B, e2_B, w_B, m_B (per source).  xi = G/K where K > 0, else 0.
int orc_canon_adjoint(long nA, const float* xA, const float* yA, const float* zA, const float* valA,
                      const float* wA, long nB, const float* xB, const float* yB, const float* zB,
                      const float* e1B, const float* e2B, const float* wB, const float* mB, const double* e2,
                      int nb, const double* lt, const double* lx, int num_threads, double* g_val, double* g_wA,
                      double* g_e1, double* g_e2, double* g_wB, double* g_m) {
  std::vector<double> sums((size_t)canon::NQ * nb, 0.0);
  orc_canon_pairs(0, nA, xA, yA, zA, valA, wA, nB, xB, yB, zB, e1B, e2B, wB, mB, e2, nb, num_threads,
                  sums.data(), nullptr, 0, nullptr);
  std::vector<double> mu(nb, 0.0), mux(nb, 0.0), nu(nb, 0.0);
  for (int b = 0; b < nb; ++b) {
    const double K = sums[canon::Q_K * nb + b];
    if (K > 0) {
      mu[b] = lt[b] / K;
      mux[b] = lx[b] / K;
      nu[b] = (lt[b] * (sums[canon::Q_GT * nb + b] / K) + lx[b] * (sums[canon::Q_GX * nb + b] / K)) / K;
    }
  }
  auto pair = [&](long i, long j, int& b, double& c2, double& s2) -> bool {
    if (wA[i] == 0.0f || zA[i] < 0.0f || zB[j] < 0.0f || zA[i] > zB[j]) return false;
    const double d2 = canon::d2_of(xA[i], yA[i], xB[j], yB[j]);
    b = canon::bin_of(d2, e2, nb);
    if (b < 0) return false;
    const double dx = (double)xA[i] - (double)xB[j], dy = (double)yA[i] - (double)yB[j];
    const double d = sqrt(d2);
    c2 = 2.0 * ((dx / d) * (dx / d)) - 1.0;
    s2 = 2.0 * dx * dy / d2;
    return true;
  };
#pragma omp parallel for schedule(dynamic, 16) num_threads(num_threads)
  for (long i = 0; i < nA; ++i) {
    double gv = 0, gw = 0;
    for (long j = 0; j < nB; ++j) {
      int b;
      double c2, s2;
      if (!pair(i, j, b, c2, s2)) continue;
      const double e1 = e1B[j], ee2 = e2B[j], w = wB[j], m = mB ? mB[j] : 0.0;
      const double t = -(e1 * c2 + ee2 * s2), x = -(-e1 * s2 + ee2 * c2);
      const double a = mu[b] * t + mux[b] * x;
      gv += a * w * (double)wA[i];
      gw += a * w * (double)valA[i] - nu[b] * w * (1.0 + m);
    }
    g_val[i] = gv;
    g_wA[i] = gw;
  }
#pragma omp parallel for schedule(dynamic, 16) num_threads(num_threads)
  for (long j = 0; j < nB; ++j) {
    double ge1 = 0, ge2 = 0, gw = 0, gm = 0;
    const double e1 = e1B[j], ee2 = e2B[j], w = wB[j], m = mB ? mB[j] : 0.0;
    for (long i = 0; i < nA; ++i) {
      int b;
      double c2, s2;
      if (!pair(i, j, b, c2, s2)) continue;
      const double vw = (double)valA[i] * (double)wA[i];
      const double t = -(e1 * c2 + ee2 * s2), x = -(-e1 * s2 + ee2 * c2);
      ge1 += (mu[b] * (-c2) + mux[b] * s2) * w * vw;
      ge2 += (mu[b] * (-s2) + mux[b] * (-c2)) * w * vw;
      gw += (mu[b] * t + mux[b] * x) * vw - nu[b] * (1.0 + m) * (double)wA[i];
      gm += -nu[b] * w * (double)wA[i];
    }
    g_e1[j] = ge1;
    g_e2[j] = ge2;
    g_wB[j] = gw;
    g_m[j] = gm;
  }
  return 0;
}

// The gradient of orc_canon_adjoint for selected objects only, given the
// per-bin totals sum_gt, sum_gx, sum_K of the whole catalogue pair (which a
// caller may take from a full-size run): each selected lens against every
// source, each selected source against every lens, in FP64 with the
// canonical bins.  Outputs are [n_lsel] and [n_ssel].
int orc_canon_adjoint_sel(long nA, const float* xA, const float* yA, const float* zA, const float* valA,
                          const float* wA, long nB, const float* xB, const float* yB, const float* zB,
                          const float* e1B, const float* e2B, const float* wB, const float* mB, const double* e2,
                          int nb, const double* sgt, const double* sgx, const double* sK, const double* lt,
                          const double* lx, const long* lsel, long n_lsel, const long* ssel, long n_ssel,
                          int num_threads, double* g_val, double* g_wA, double* g_e1, double* g_e2, double* g_wB,
                          double* g_m) {
  std::vector<double> mu(nb, 0.0), mux(nb, 0.0), nu(nb, 0.0);
  for (int b = 0; b < nb; ++b) {
    const double K = sK[b];
    if (K > 0) {
      mu[b] = lt[b] / K;
      mux[b] = lx[b] / K;
      nu[b] = (lt[b] * (sgt[b] / K) + lx[b] * (sgx[b] / K)) / K;
    }
  }
  auto pair = [&](long i, long j, int& b, double& c2, double& s2) -> bool {
    if (wA[i] == 0.0f || zA[i] < 0.0f || zB[j] < 0.0f || zA[i] > zB[j]) return false;
    const double d2 = canon::d2_of(xA[i], yA[i], xB[j], yB[j]);
    b = canon::bin_of(d2, e2, nb);
    if (b < 0) return false;
    const double dx = (double)xA[i] - (double)xB[j], dy = (double)yA[i] - (double)yB[j];
    const double d = sqrt(d2);
    c2 = 2.0 * ((dx / d) * (dx / d)) - 1.0;
    s2 = 2.0 * dx * dy / d2;
    return true;
  };
#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads)
  for (long k = 0; k < n_lsel; ++k) {
    const long i = lsel[k];
    double gv = 0, gw = 0;
    for (long j = 0; j < nB; ++j) {
      int b;
      double c2, s2;
      if (!pair(i, j, b, c2, s2)) continue;
      const double e1 = e1B[j], ee2 = e2B[j], w = wB[j], m = mB ? mB[j] : 0.0;
      const double t = -(e1 * c2 + ee2 * s2), x = -(-e1 * s2 + ee2 * c2);
      const double a = mu[b] * t + mux[b] * x;
      gv += a * w * (double)wA[i];
      gw += a * w * (double)valA[i] - nu[b] * w * (1.0 + m);
    }
    g_val[k] = gv;
    g_wA[k] = gw;
  }
  for (long k = 0; k < n_ssel; ++k) {
    const long j = ssel[k];
    const double e1 = e1B[j], ee2 = e2B[j], w = wB[j], m = mB ? mB[j] : 0.0;
    double ge1 = 0, ge2 = 0, gw = 0, gm = 0;
#pragma omp parallel for schedule(static) num_threads(num_threads) reduction(+ : ge1, ge2, gw, gm)
    for (long i = 0; i < nA; ++i) {
      int b;
      double c2, s2;
      if (!pair(i, j, b, c2, s2)) continue;
      const double vw = (double)valA[i] * (double)wA[i];
      const double t = -(e1 * c2 + ee2 * s2), x = -(-e1 * s2 + ee2 * c2);
      ge1 += (mu[b] * (-c2) + mux[b] * s2) * w * vw;
      ge2 += (mu[b] * (-s2) + mux[b] * (-c2)) * w * vw;
      gw += (mu[b] * t + mux[b] * x) * vw - nu[b] * (1.0 + m) * (double)wA[i];
      gm += -nu[b] * w * (double)wA[i];
    }
    g_e1[k] = ge1;
    g_e2[k] = ge2;
    g_wB[k] = gw;
    g_m[k] = gm;
  }
  return 0;
}

// ------------------------------------------------------------ spherical --
// Reference restatement in FP32 (src/utils.f90:512-528 distance_sphere,
// :618-639 angles_sphere; pair loop src/tpcf.f90:297-359 with
// spherical_coords, all pairs, no kd-tree), and the canonical FP64 rule the
// library uses on the sphere: chord^2 = |u_B - u_A|^2 of unit vectors from
// FP64 sin/cos of the FP32 (lambda, phi) in radians, against squared chords
// (2 sin(e/2))^2 of the FP64 edges; position angle from A = du.east_A,
// B = du.north_A (the numerators of angles_sphere).
static inline float distance_sphere_f32(float l1, float p1, float l2, float p2) {
  float cos_d = sinf(p1) * sinf(p2) + cosf(p1) * cosf(p2) * cosf(l2 - l1);
  if (cos_d >= 1.0f) return 0.0f;
  if (cos_d <= -1.0f) return 3.141592653589793f;
  return acosf(cos_d);
}

int orc_ref_sphere_f32(int mode, long nA, const float* xA, const float* yA, const float* zA, const float* valA,
                       const float* wA, long nB, const float* xB, const float* yB, const float* zB,
                       const float* e1B, const float* e2B, const float* wB, const float* mB, float x_min,
                       float x_max, int n_bin, int spacing, float p, int num_threads, float* g_t, float* g_x,
                       float* weights, long long* n_pairs) {
  ref::Binning<float> b;
  if (ref::create_bins<float>(x_min, x_max, n_bin, spacing, p, b)) return 10;
  std::vector<float> gt(n_bin, 0), gx(n_bin, 0), W(n_bin, 0), K(n_bin, 0);
  std::vector<long long> np(n_bin, 0);
#pragma omp parallel num_threads(num_threads)
  {
    std::vector<float> lgt(n_bin, 0), lgx(n_bin, 0), lw(n_bin, 0), lK(n_bin, 0);
    std::vector<long long> lnp(n_bin, 0);
#pragma omp for schedule(static)
    for (long i = 0; i < nA; ++i) {
      const float l1 = xA[i], p1 = yA[i], vf = valA[i], wf = wA[i];
      const float zf = mode == 0 ? zA[i] : 0.0f;
      if (wf == 0.0f) continue;
      for (long j = 0; j < nB; ++j) {
        if (mode == 0 && (zf < 0.0f || zB[j] < 0.0f || zf > zB[j])) continue;
        const float l2 = xB[j], p2 = yB[j];
        const float dist = distance_sphere_f32(l1, p1, l2, p2);
        const int bi = ref::find_bin_index(dist, b);
        if (bi < 0) continue;
        const float w = wB[j];
        if (mode == 0) {
          const float sin_d = sinf(dist), cos_p2 = cosf(p2);
          const float cs1 = cos_p2 / sin_d * sinf(l2 - l1);
          const float cs2 = (cosf(p1) * sinf(p2) - sinf(p1) * cos_p2 * cosf(l2 - l1)) / sin_d;
          const float c2 = 2.0f * cs1 * cs1 - 1.0f, s2 = 2.0f * cs1 * cs2;
          const float e1 = e1B[j], e2 = e2B[j], m = mB ? mB[j] : 0.0f;
          lgt[bi] -= (e1 * c2 + e2 * s2) * w * vf * wf;
          lgx[bi] -= (-e1 * s2 + e2 * c2) * w * vf * wf;
          lK[bi] += w * (1.0f + m) * wf;
        } else {
          lgt[bi] += e1B[j] * w * vf * wf;
          lgx[bi] += e2B[j] * w * vf * wf;
          lK[bi] += w * wf;
        }
        lw[bi] += w * wf;
        lnp[bi] += 1;
      }
    }
#pragma omp critical
    for (int q = 0; q < n_bin; ++q) {
      gt[q] += lgt[q]; gx[q] += lgx[q]; W[q] += lw[q]; K[q] += lK[q]; np[q] += lnp[q];
    }
  }
  for (int q = 0; q < n_bin; ++q) {
    g_t[q] = K[q] > 0 ? gt[q] / K[q] : 0.0f;
    g_x[q] = K[q] > 0 ? gx[q] / K[q] : 0.0f;
    weights[q] = W[q];
    n_pairs[q] = np[q];
  }
  return 0;
}

// Canonical unit vectors on the sphere: sin/cos in FP64 by one fixed
// sequence of rounded operations (Cody-Waite reduction by pi/2 in three
// parts, Taylor series through r^17 / r^18), u = (cos phi cos lambda,
// cos phi sin lambda, sin phi), hi = fl32(u), lo = fl32(u - hi).  This file
// is built with -ffp-contract=off, so every operation rounds as written.
namespace sph {
static void sincos_fixed(double x, double& s, double& c) {
  const double two_over_pi = 0.6366197723675814;
  const double p1 = 1.5707963267341256, p2 = 6.077100506303966e-11, p3 = 2.0222662487959506e-21;
  const double k = std::rint(x * two_over_pi);
  double r = x - k * p1;
  r = r - k * p2;
  r = r - k * p3;
  const double z = r * r;
  // 1/n! for odd n = 17, 15, ..., 3 and even n = 18, 16, ..., 4
  const double so[8] = {2.8114572543455206e-15, 7.647163731819816e-13, 1.6059043836821613e-10,
                        2.505210838544172e-08, 2.7557319223985893e-06, 0.0001984126984126984,
                        0.008333333333333333, 0.16666666666666666};
  const double ce[8] = {4.779477332387385e-14, 1.1470745597729725e-11, 2.08767569878681e-09,
                        2.755731922398589e-07, 2.48015873015873e-05, 0.001388888888888889,
                        0.041666666666666664};
  double ps = so[0];
  for (int i = 1; i < 8; ++i) ps = (i % 2) ? ps * z - so[i] : ps * z + so[i];
  const double sr = r + (r * z) * ps;
  double pc = -1.5619206968586225e-16;
  for (int i = 0; i < 7; ++i) pc = (i % 2) ? pc * z - ce[i] : pc * z + ce[i];
  const double cr = 1.0 + (-0.5 * z + (z * z) * pc);
  switch ((int)((long long)k & 3)) {
    case 0: s = sr; c = cr; break;
    case 1: s = cr; c = -sr; break;
    case 2: s = -sr; c = -cr; break;
    default: s = -cr; c = sr; break;
  }
}
static void unit_hilo(float lam, float phi, float hi[3], float lo[3]) {
  double sl, cl, sp, cp;
  sincos_fixed((double)lam, sl, cl);
  sincos_fixed((double)phi, sp, cp);
  const double u[3] = {cp * cl, cp * sl, sp};
  for (int k = 0; k < 3; ++k) {
    hi[k] = (float)u[k];
    lo[k] = (float)(u[k] - (double)hi[k]);
  }
}
}  // namespace sph

int orc_unit_vectors(long n, const float* lam, const float* phi, float* hi, float* lo) {
  for (long i = 0; i < n; ++i) sph::unit_hilo(lam[i], phi[i], hi + 3 * i, lo + 3 * i);
  return 0;
}

// Canonical FP64 spherical sums, [8][n_bin] as orc_canon_pairs (the dw row
// is theta * w_B * w_A with theta = 2 asin(chord/2)).  e2 are the squared
// canonical chords (orc_sphere_edges_sq).  Chord^2 from u = hi + lo in FP64:
// (dx*dx + dy*dy) + dz*dz with d = u_B - u_A.  Position angle at the lens
// from A = d.east, B = d.north with the lens frame from libm sin/cos (an
// independent evaluation of angles_sphere, src/utils.f90:618-639).
int orc_canon_sphere(int mode, long nA, const float* xA, const float* yA, const float* zA, const float* valA,
                     const float* wA, long nB, const float* xB, const float* yB, const float* zB,
                     const float* e1B, const float* e2B, const float* wB, const float* mB, const double* e2,
                     int nb, int num_threads, double* sums) {
  const int NQ = canon::NQ;
  std::vector<double> ub(3 * (size_t)nB);
  for (long j = 0; j < nB; ++j) {
    float h[3], l[3];
    sph::unit_hilo(xB[j], yB[j], h, l);
    for (int k = 0; k < 3; ++k) ub[3 * j + k] = (double)h[k] + (double)l[k];
  }
  const long CH = 64;
  const long nch = (nA + CH - 1) / CH;
  std::vector<double> part((size_t)nch * NQ * nb, 0.0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads)
  for (long c = 0; c < nch; ++c) {
    double* acc = part.data() + (size_t)c * NQ * nb;
    for (long i = c * CH; i < std::min(nA, (c + 1) * CH); ++i) {
      if (wA[i] == 0.0f || (mode == 0 && zA[i] < 0.0f)) continue;
      float h[3], l[3];
      sph::unit_hilo(xA[i], yA[i], h, l);
      const double ua[3] = {(double)h[0] + (double)l[0], (double)h[1] + (double)l[1], (double)h[2] + (double)l[2]};
      const double lam = xA[i], ph = yA[i];
      const double east[3] = {-sin(lam), cos(lam), 0.0};
      const double north[3] = {-sin(ph) * cos(lam), -sin(ph) * sin(lam), cos(ph)};
      const double vw = (double)valA[i] * (double)wA[i];
      for (long j = 0; j < nB; ++j) {
        if (mode == 0 && (zB[j] < 0.0f || zA[i] > zB[j])) continue;
        const double d0 = ub[3 * j] - ua[0], d1 = ub[3 * j + 1] - ua[1], d2c = ub[3 * j + 2] - ua[2];
        const double ch2 = (d0 * d0 + d1 * d1) + d2c * d2c;
        const int b = canon::bin_of(ch2, e2, nb);
        if (b < 0) continue;
        const double w = wB[j];
        const double ang = 2.0 * asin(sqrt(ch2) / 2.0);
        double tt, tx, kk;
        if (mode == 0) {
          const double A = d0 * east[0] + d1 * east[1] + d2c * east[2];
          const double B = d0 * north[0] + d1 * north[1] + d2c * north[2];
          const double s = A * A + B * B;
          const double c2 = (A * A - B * B) / s, s2 = 2.0 * A * B / s;
          const double e1 = e1B[j], ee2 = e2B[j];
          tt = -(e1 * c2 + ee2 * s2) * w * vw;
          tx = -(-e1 * s2 + ee2 * c2) * w * vw;
          kk = w * (1.0 + (mB ? (double)mB[j] : 0.0)) * (double)wA[i];
        } else {
          tt = (double)e1B[j] * w * vw;
          tx = (double)e2B[j] * w * vw;
          kk = w * (double)wA[i];
        }
        acc[canon::Q_DW * nb + b] += ang * w * (double)wA[i];
        acc[canon::Q_GT * nb + b] += tt;
        acc[canon::Q_GX * nb + b] += tx;
        acc[canon::Q_W * nb + b] += w * (double)wA[i];
        acc[canon::Q_K * nb + b] += kk;
        acc[canon::Q_N * nb + b] += 1.0;
        acc[canon::Q_AGT * nb + b] += fabs(tt);
        acc[canon::Q_AGX * nb + b] += fabs(tx);
        const double nt = mode == 0 ? hypot((double)e1B[j], (double)e2B[j]) * w * fabs(vw) : fabs(tt);
        acc[canon::Q_NGT * nb + b] += nt;
        acc[canon::Q_NGX * nb + b] += mode == 0 ? nt : fabs(tx);
      }
    }
  }
  std::fill(sums, sums + (size_t)NQ * nb, 0.0);
  for (long c = 0; c < nch; ++c)
    for (int q = 0; q < NQ * nb; ++q) sums[q] += part[(size_t)c * NQ * nb + q];
  return 0;
}

// Squared canonical chords of the FP64 angle edges: (2 sin(e/2))^2 with the
// fixed sine above.
int orc_sphere_edges_sq(const double* edges, int nb, double* out) {
  for (int i = 0; i <= nb; ++i) {
    double s, c;
    sph::sincos_fixed(edges[i] * 0.5, s, c);
    const double ch = 2.0 * s;
    out[i] = ch * ch;
  }
  return 0;
}

// rotate_data_from_poles_and_meridian (src/main.f90:953-1015) with
// rotation_sphere (src/utils.f90:483-509), distance_to_meridian_sphere
// (:579-599) and median (:712-726), all in FP32 as the reference compiles
// them.  In place.
namespace rot {
const float PI = 3.141592653589793f;
static float dist_meridian(float l1, float p1, float l2) {
  const float sd = fabsf(sinf(l2 - l1) * cosf(p1));
  if (fabsf(l2 - l1) <= PI / 2.0f) return sd >= 1.0f ? PI / 2.0f : asinf(sd);
  return PI / 2.0f - fabsf(p1);
}
static float kth(std::vector<float> v, long k1) {  // k1-th smallest, 1-based
  std::nth_element(v.begin(), v.begin() + (k1 - 1), v.end());
  return v[k1 - 1];
}
static float median(const float* x, long n) {
  std::vector<float> v(x, x + n);
  if (n % 2 == 0) return (kth(v, n / 2 + 1) + kth(v, n / 2)) / 2.0f;
  return kth(v, n / 2 + 1);
}
static void rotation(float& lam, float& phi, float lam_rot, float phi_rot) {
  const float sigma = lam + lam_rot;
  const float theta = PI / 2.0f - phi;
  const float theta_rot = -phi_rot;
  const float x = cosf(sigma) * cosf(theta_rot) * sinf(theta) + cosf(theta) * sinf(theta_rot);
  const float y = sinf(sigma) * sinf(theta);
  const float z = -cosf(sigma) * sinf(theta_rot) * sinf(theta) + cosf(theta) * cosf(theta_rot);
  float lo = atanf(y / x);
  if (x < 0.0f) lo = lo + PI;
  float po;
  if (z >= 1.0f) po = PI / 2.0f;
  else if (z <= -1.0f) po = -PI / 2.0f;
  else po = PI / 2.0f - acosf(z);
  lam = lo;
  phi = po;
}
}  // namespace rot

int orc_rotate_from_poles(float* xA, float* yA, long nA, float* xB, float* yB, long nB, float r_max, int* rotated,
                          float* center) {
  using namespace rot;
  auto mn = [](const float* v, long n) { return *std::min_element(v, v + n); };
  auto mx = [](const float* v, long n) { return *std::max_element(v, v + n); };
  float x_min = mn(xA, nA), x_max = mx(xA, nA), y_min = mn(yA, nA), y_max = mx(yA, nA);
  bool r = false;
  if (y_max + r_max >= PI / 2.0f) r = true;
  else if (y_min - r_max <= -PI / 2.0f) r = true;
  if (x_max - x_min > PI) {
    for (long i = 0; i < nA; ++i)
      if (xA[i] > PI) xA[i] = xA[i] - 2.0f * PI;
    x_min = mn(xA, nA);
    x_max = mx(xA, nA);
    r = true;
  } else if (dist_meridian(x_max, y_max, 0.0f) <= r_max || dist_meridian(x_min, y_max, 0.0f) <= r_max ||
             dist_meridian(x_max, y_min, 0.0f) <= r_max || dist_meridian(x_min, y_min, 0.0f) <= r_max) {
    r = true;
  }
  if (xB && nB > 0 && mx(xB, nB) - mn(xB, nB) > PI)
    for (long i = 0; i < nB; ++i)
      if (xB[i] > PI) xB[i] = xB[i] - 2.0f * PI;
  center[0] = center[1] = 0.0f;
  if (r) {
    const float cx = median(xA, nA), cy = median(yA, nA);
    center[0] = cx;
    center[1] = cy;
    for (long i = 0; i < nA; ++i) rotation(xA[i], yA[i], PI - cx, -cy);
    if (xB)
      for (long i = 0; i < nB; ++i) rotation(xB[i], yB[i], PI - cx, -cy);
  }
  *rotated = r ? 1 : 0;
  return 0;
}

// kd-tree radius search (test_kdtree.f90).  Results are 0-based indices.
int orc_kdtree_search(long n, const float* x, const float* y, float qx, float qy, float r,
                      int leafsize, int brute_force, long* results, long cap, long* n_found) {
  ref::KDTree<float> t;
  if (t.grow(x, y, n, leafsize)) return 3;
  long nf = 0;
  int e = t.search(qx, qy, r, results, cap, nf, brute_force != 0);
  for (long i = 0; i < std::min(nf, cap); ++i) results[i] -= 1;
  *n_found = nf;
  return e;
}

int orc_kmeans_ref_f32(long n, const float* x, const float* y, const float* w, int k,
                       int equal_size, float scaling, int max_iter, float reassign_tol,
                       float weight_tol, int* labels, float* cx, float* cy, int* n_iter) {
  return ref::partition_data<float>(n, x, y, w, k, equal_size != 0, scaling, max_iter,
                                    reassign_tol, weight_tol, labels, cx, cy, n_iter);
}

int orc_qsort_arg_f32(const float* a, long n, long* order, int reverse) {
  ref::qsort_arg(a, n, order, reverse != 0);
  return 0;
}

// Deterministic Voronoi-mode k-means as the CUDA library defines it: the same
// fixed-grid start as kmeans.f90:85-112 (FP32), FP32 IEEE distances
// sqrt(dx*dx+dy*dy) compared with a strict '<' from index 0 upward, and
// centroids from fixed-point (int64) sums of x*w and w, so that the result is
// independent of summation order.  Labels 0-based.
int orc_kmeans_det(long n, const float* x, const float* y, const float* w, int k, int max_iter,
                   float reassign_tol, int* labels, float* cx, float* cy, int* n_iter_out) {
  if (k <= 1 || n < 1) return 1;
  float xmn = x[0], xmx = x[0], ymn = y[0], ymx = y[0];
  double amax = 0, wmax = 0;
  for (long i = 0; i < n; ++i) {
    xmn = std::min(xmn, x[i]); xmx = std::max(xmx, x[i]);
    ymn = std::min(ymn, y[i]); ymx = std::max(ymx, y[i]);
    wmax = std::max(wmax, fabs((double)w[i]));
  }
  amax = std::max(std::max(fabs((double)xmn), fabs((double)xmx)), std::max(fabs((double)ymn), fabs((double)ymx)));
  float diam = sqrtf((xmx - xmn) * (xmx - xmn) + (ymx - ymn) * (ymx - ymn));
  int n_side = (int)sqrtf((float)k);
  if (xmx - xmn > ymx - ymn) {
    float dy = (ymx - ymn) / (float)n_side;
    float dx = (xmx - xmn) * (float)n_side / (float)k;
    for (int j = 1; j <= k; ++j) {
      int row = (int)((dx / 2.0f + dx * (float)(j - 1)) / (xmx - xmn));
      cx[j - 1] = xmn + fmodf(dx / 2.0f + dx * (float)(j - 1), xmx - xmn);
      cy[j - 1] = ymn + dy / 2.0f + dy * (float)row;
    }
  } else {
    float dx = (xmx - xmn) / (float)n_side;
    float dy = (ymx - ymn) * (float)n_side / (float)k;
    for (int j = 1; j <= k; ++j) {
      int row = (int)((dy / 2.0f + dy * (float)(j - 1)) / (ymx - ymn));
      cy[j - 1] = ymn + fmodf(dy / 2.0f + dy * (float)(j - 1), ymx - ymn);
      cx[j - 1] = xmn + dx / 2.0f + dx * (float)row;
    }
  }
  for (long i = 0; i < n; ++i) labels[i] = (int)((float)i / (float)n * (float)k + 1.0f) - 1;
  const int sp = det::fixed_scale(n, amax * wmax);
  const int sw = det::fixed_scale(n, wmax);
  int it = 0;
  while (it <= max_iter) {
    ++it;
    long n_re = 0;
    for (long i = 0; i < n; ++i) {
      float min_d = diam * 10.0f;
      int ci = -1;
      for (int j = 0; j < k; ++j) {
        float ddx = x[i] - cx[j], ddy = y[i] - cy[j];
        float d = sqrtf(ddx * ddx + ddy * ddy);
        if (d < min_d) { min_d = d; ci = j; }
      }
      if (ci != labels[i]) { labels[i] = ci; ++n_re; }
    }
    std::vector<long long> ax(k, 0), ay(k, 0), aw(k, 0);
    for (long i = 0; i < n; ++i) {
      int c = labels[i];
      if (c < 0) continue;
      ax[c] += llrint(ldexp((double)x[i] * (double)w[i], sp));
      ay[c] += llrint(ldexp((double)y[i] * (double)w[i], sp));
      aw[c] += llrint(ldexp((double)w[i], sw));
    }
    for (int j = 0; j < k; ++j) {
      double W = ldexp((double)aw[j], -sw);
      cx[j] = (float)(ldexp((double)ax[j], -sp) / W);
      cy[j] = (float)(ldexp((double)ay[j], -sp) / W);
    }
    if (n_re == 0) break;
    if ((float)n_re / (float)n < reassign_tol) break;
  }
  if (n_iter_out) *n_iter_out = it;
  return 0;
}

// Equal-weight k-means (partition_data with equal_size, src/kmeans.f90:12-262)
// restated serially with the library's deterministic choices: the points are
// swept in order in chunks (32..1024 points, n/2048) and the points of a chunk
// see the cluster weights the previous chunks left (the reference moves the
// weight of each reassigned point at once, in OpenMP thread order);
// fixed-point weights and sums; Philox draws for the random start.  The rebalance follows
// postprocess_weights (:221-262) point by point.
int orc_kmeans_equal_det(long n, const float* x, const float* y, const float* w, int k, int max_iter,
                         float reassign_tol, float scaling, float weight_tol, int random_init, uint64_t seed,
                         int* labels, float* cx, float* cy, int* n_iter_out, float* max_dev_out) {
  if (k <= 1 || n < 1) return 1;
  float xmn = x[0], xmx = x[0], ymn = y[0], ymx = y[0];
  double wmax = 0;
  for (long i = 0; i < n; ++i) {
    xmn = std::min(xmn, x[i]); xmx = std::max(xmx, x[i]);
    ymn = std::min(ymn, y[i]); ymx = std::max(ymx, y[i]);
    wmax = std::max(wmax, fabs((double)w[i]));
  }
  const double amax = std::max(std::max(fabs((double)xmn), fabs((double)xmx)), std::max(fabs((double)ymn), fabs((double)ymx)));
  const float diam = sqrtf((xmx - xmn) * (xmx - xmn) + (ymx - ymn) * (ymx - ymn));
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  if (random_init) {
    std::vector<long> chosen;
    for (uint32_t t = 0; (int)chosen.size() < k; ++t) {
      uint32_t c[4] = {t / 4, 0xC3u, 0x4B4Du, 0u};
      det::philox4x32(c, k0, k1);
      const long idx = (long)(((uint64_t)c[t % 4] * (uint64_t)n) >> 32);
      if (std::find(chosen.begin(), chosen.end(), idx) == chosen.end()) chosen.push_back(idx);
    }
    for (int j = 0; j < k; ++j) { cx[j] = x[chosen[j]]; cy[j] = y[chosen[j]]; }
    for (long q = 0; q < (n + 3) / 4; ++q) {
      uint32_t c[4] = {(uint32_t)q, 0xC4u, 0x4B4Du, 0u};
      det::philox4x32(c, k0, k1);
      for (int u = 0; u < 4; ++u)
        if (4 * q + u < n) labels[4 * q + u] = (int)(((uint64_t)c[u] * (uint32_t)k) >> 32);
    }
  } else {
    int n_side = (int)sqrtf((float)k);
    if (xmx - xmn > ymx - ymn) {
      float dy = (ymx - ymn) / (float)n_side;
      float dx = (xmx - xmn) * (float)n_side / (float)k;
      for (int j = 1; j <= k; ++j) {
        int row = (int)((dx / 2.0f + dx * (float)(j - 1)) / (xmx - xmn));
        cx[j - 1] = xmn + fmodf(dx / 2.0f + dx * (float)(j - 1), xmx - xmn);
        cy[j - 1] = ymn + dy / 2.0f + dy * (float)row;
      }
    } else {
      float dx = (xmx - xmn) / (float)n_side;
      float dy = (ymx - ymn) * (float)n_side / (float)k;
      for (int j = 1; j <= k; ++j) {
        int row = (int)((dy / 2.0f + dy * (float)(j - 1)) / (ymx - ymn));
        cy[j - 1] = ymn + fmodf(dy / 2.0f + dy * (float)(j - 1), ymx - ymn);
        cx[j - 1] = xmn + dx / 2.0f + dx * (float)row;
      }
    }
    for (long i = 0; i < n; ++i) labels[i] = (int)((float)i / (float)n * (float)k + 1.0f) - 1;
  }
  const int sp = det::fixed_scale(n, amax * wmax);
  const int sw = det::fixed_scale(n, wmax);
  std::vector<long long> W(k, 0);
  for (long i = 0; i < n; ++i)
    if (labels[i] >= 0) W[labels[i]] += llrint(ldexp((double)w[i], sw));
  long long tot = 0;
  for (int j = 0; j < k; ++j) tot += W[j];
  const float wmean = (float)(ldexp((double)tot, -sw) / k);
  const long chunk = std::max(32L, std::min(1024L, n / 2048));
  std::vector<int> cand(n, -1);
  std::vector<float> memb(n, 0.0f), f(k, 1.0f);
  int it = 0;
  while (it <= max_iter) {
    ++it;
    const bool pen = it > 1 && scaling > 0.0f, cands = it > 1;
    long n_re = 0;
    for (long base = 0; base < n; base += chunk) {
      // the points of one chunk see the weights the previous chunks left
      for (int j = 0; j < k; ++j)
        f[j] = pen ? 1.0f + (((float)ldexp((double)W[j], -sw) / wmean) - 1.0f) * scaling : 1.0f;
      for (long i = base; i < std::min(n, base + chunk); ++i) {
        float best = diam * 10.0f, cm = 0.0f;
        int bi = -1, ci = -1;
        for (int j = 0; j < k; ++j) {
          const float ddx = x[i] - cx[j], ddy = y[i] - cy[j];
          const float d = f[j] * sqrtf(ddx * ddx + ddy * ddy);
          if (cands && d > 0.0f) {
            if (d < best) { cm = best / d; ci = bi; best = d; bi = j; }
            else if (d < cm * best) { cm = d / best; ci = j; }
          } else if (d < best) { best = d; bi = j; }
        }
        if (cands) { cand[i] = ci; memb[i] = cm; }
        const int old = labels[i];
        if (bi != old) {
          labels[i] = bi;
          ++n_re;
          const long long wf = llrint(ldexp((double)w[i], sw));
          if (old >= 0) W[old] -= wf;
          if (bi >= 0) W[bi] += wf;
        }
      }
    }
    std::vector<long long> ax(k, 0), ay(k, 0), aw(k, 0);
    for (long i = 0; i < n; ++i) {
      const int c = labels[i];
      if (c < 0) continue;
      ax[c] += llrint(ldexp((double)x[i] * (double)w[i], sp));
      ay[c] += llrint(ldexp((double)y[i] * (double)w[i], sp));
      aw[c] += llrint(ldexp((double)w[i], sw));
    }
    for (int j = 0; j < k; ++j) {
      const double Wd = ldexp((double)aw[j], -sw);
      cx[j] = (float)(ldexp((double)ax[j], -sp) / Wd);
      cy[j] = (float)(ldexp((double)ay[j], -sp) / Wd);
    }
    if (n_re == 0) break;
    if ((float)n_re / (float)n < reassign_tol) break;
  }
  auto max_dev = [&]() {
    const long long mx = *std::max_element(W.begin(), W.end()), mn = *std::min_element(W.begin(), W.end());
    return (float)(ldexp((double)(mx - mn), -sw) / (double)wmean);
  };
  float dev = max_dev();
  if (dev > weight_tol && it > 1) {
    std::vector<int> corder(k);
    for (int j = 0; j < k; ++j) corder[j] = j;
    std::stable_sort(corder.begin(), corder.end(), [&](int a, int b) { return W[a] > W[b]; });
    std::vector<long> order(n);
    for (long i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](long a, long b) { return memb[a] < memb[b]; });
    const long long thr = llrint(ldexp((double)(wmean * (1.0f + weight_tol)), sw));
    std::vector<char> done(k, 0);
    for (int j = 0; j < k; ++j) {
      const int cj = corder[j];
      done[cj] = 1;
      for (long r = 0; r < n; ++r) {
        const long p = order[r];
        const int d = cand[p];
        if (labels[p] != cj || d < 0 || done[d]) continue;
        const long long wf = llrint(ldexp((double)w[p], sw));
        labels[p] = d;
        W[cj] -= wf;
        W[d] += wf;
        if (W[cj] <= thr) break;
      }
    }
    dev = max_dev();
  }
  if (n_iter_out) *n_iter_out = it;
  if (max_dev_out) *max_dev_out = dev;
  return 0;
}

int orc_fixed_scale(long n, double vmax) { return det::fixed_scale(n, vmax); }

// Raw Philox4x32-10 block, for known-answer tests.
void orc_philox4x32(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  det::philox4x32(c, key[0], key[1]);
  for (int i = 0; i < 4; ++i) out[i] = c[i];
}

// Multiplicity matrix [n_boot][n_patch] from n_draw Philox draws per sample.
int orc_bootstrap_multiplicity(uint64_t seed, int n_boot, int n_patch, int n_draw, int* mult) {
  std::fill(mult, mult + (size_t)n_boot * n_patch, 0);
  for (int s = 0; s < n_boot; ++s)
    for (int d = 0; d < n_draw; ++d) mult[(size_t)s * n_patch + det::draw(seed, s, d, n_patch)] += 1;
  return 0;
}

// Block bootstrap from patch sums, src/tpcf.f90:1166-1191 restated in FP64.
//   St, Sx, SK: [n_patch][n_bin]; Sw: [n_patch]; mult: [n_boot][n_patch]
int orc_block_bootstrap(int n_boot, int n_patch, int n_bin, const int* mult, const double* St,
                        const double* Sx, const double* SK, const double* Sw, double* gt,
                        double* gx, double* weights) {
  for (int s = 0; s < n_boot; ++s) {
    double W = 0;
    for (int b = 0; b < n_bin; ++b) {
      double t = 0, x = 0, K = 0;
      for (int p = 0; p < n_patch; ++p) {
        double m = mult[(size_t)s * n_patch + p];
        t += St[(size_t)p * n_bin + b] * m;
        x += Sx[(size_t)p * n_bin + b] * m;
        K += SK[(size_t)p * n_bin + b] * m;
      }
      gt[(size_t)s * n_bin + b] = K > 0 ? t / K : 0.0;
      gx[(size_t)s * n_bin + b] = K > 0 ? x / K : 0.0;
    }
    for (int p = 0; p < n_patch; ++p) W += Sw[p] * mult[(size_t)s * n_patch + p];
    weights[s] = W;
  }
  return 0;
}

// covariance_matrix, src/utils.f90:745-764, in FP64.  x is [n_samples][n_data].
int orc_covariance(int n_samples, int n_data, const double* x, double* cov) {
  for (int i = 0; i < n_data; ++i) {
    double mi = 0;
    for (int s = 0; s < n_samples; ++s) mi += x[(size_t)s * n_data + i];
    mi /= n_samples;
    for (int j = 0; j <= i; ++j) {
      double mj = 0;
      for (int s = 0; s < n_samples; ++s) mj += x[(size_t)s * n_data + j];
      mj /= n_samples;
      double c = 0;
      for (int s = 0; s < n_samples; ++s)
        c += (x[(size_t)s * n_data + i] - mi) * (x[(size_t)s * n_data + j] - mj);
      c /= (n_samples - 1);
      cov[(size_t)i * n_data + j] = c;
      cov[(size_t)j * n_data + i] = c;
    }
  }
  return 0;
}

}  // extern "C"
