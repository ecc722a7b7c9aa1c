// C-ABI of the grid side of libnapmo: radial transforms, Lebedev/radial/
// atomic/Becke grids, cubic splines and extrapolations, the Hermite FEM
// assembly, and the device Poisson pipeline.  Symbol names, argument order
// and meaning follow the ctypes bindings of nAPMO (napmo/__init__.py:
// 106-585); every function that evaluates something per grid point runs on
// the GPU.
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <algorithm>
#include <vector>

#include "capi_common.cuh"
#include "host.h"
#include "kernels.cuh"
#include "poisson.cuh"
#include "solid_harmonics.h"

namespace napmo {

int last_error(char *buf, int len);

cudaStream_t host_api_stream() {
  static thread_local std::map<int, cudaStream_t> streams;
  int dev = 0;
  cudaGetDevice(&dev);
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  streams[dev] = s;
  return s;
}

// ------------------------------------------------------------ Poisson plan
struct PoissonPlan {
  PoissonDev d;
  int lmax = -1;
  int max_mol_npoint = 0;
  std::vector<PoissonAtom> h_atoms;
  DevBuf<PoissonAtom> atoms;
  DevBuf<int> mol_atom_off, mol_point_off, sys_atom, sys_l;
  DevBuf<double> rad, ytab, proj, spl, amp, raw_y, raw_dt, lu, lmul;
  DevBuf<int> lpiv;
  DevBuf<double> rscr;  // radial-solve scratch of one solve
  DevBuf<double> pg;    // projection scratch of one solve (rho wb w per point)
  DevBuf<int> pairs;
  DevBuf<double2> pair_u;  // (u, 1/d) of each interior pair
  DevBuf<EvalItem> items;
  int nitems = 0, nitems_in = 0;  // items, of which the first nitems_in are interior
  int chunk = kEvalChunk;         // pairs per item
  DevBuf<double> pair_v;
  DevBuf<int> lcut;  // per bucket, for truncated evaluations
  // pair lists of the points kept by a screening mask (built for the last
  // mask used; the mask is owned by the caller's int8 plan)
  DevBuf<int> pairs_s;
  DevBuf<double2> pair_u_s;
  DevBuf<EvalItem> items_s;
  int nitems_s = 0, nitems_in_s = 0, chunk_s = kEvalChunk;
  unsigned long long screen_key = 0;  // serial of the mask's int8 plan (0: none)
  // Becke-Dickson workspace (source, shell averages, LU factors), kept
  // between calls: an allocation per call would return to the driver at
  // every synchronisation of the caller's loop
  DevBuf<char> bd_ws;
  // per-solve tables (projection, splines, amplitudes, pair potentials,
  // truncation) of batched solves
  DevBuf<char> batch_ws;
};

void free_poisson_plan(PoissonPlan *p) { delete p; }

// Solid harmonics of the Lebedev directions: Y[j][lm], lm < (lmax+1)^2.
static void ytable(const std::vector<double> &ang, int nang, int lmax,
                   std::vector<double> &out) {
  const int lsize = (lmax + 1) * (lmax + 1);
  out.assign((size_t)nang * lsize, 0.0);
  std::vector<double> work(lsize + 3);
  for (int j = 0; j < nang; ++j) {
    double *y = &out[(size_t)j * lsize];
    y[0] = 1.0;
    if (lmax >= 1) {
      work[0] = ang[j * 3 + 2];
      work[1] = ang[j * 3 + 0];
      work[2] = ang[j * 3 + 1];
      solid_harmonics(work.data(), lmax);
      for (int k = 1; k < lsize; ++k) y[k] = work[k - 1];
    }
  }
}

int build_poisson_plan(const std::vector<const AtomLayout *> &atoms,
                       const std::vector<int> &lmax_of, const std::vector<int> &mol_atom_off,
                       const std::vector<int> &mol_point_off, cudaStream_t s,
                       PoissonPlan *plan) {
  NAPMO_TRY_CUDA(poisson_init_constants(), "poisson constants");
  const int natom = (int)atoms.size();
  PoissonDev &d = plan->d;
  d = PoissonDev();
  d.natom = natom;
  d.nmol = (int)mol_atom_off.size() - 1;
  std::vector<PoissonAtom> &ha = plan->h_atoms;
  ha.assign(natom, PoissonAtom());
  std::vector<double> rad, ytab;
  std::map<std::pair<int, int>, int> ykey;  // (atom-rule id via nang,lmax) -> offset
  std::vector<int> sys_atom, sys_l;
  long proj = 0, spl = 0, amp = 0, raw = 0, pairs = 0, scr = 0, npts = 0;
  int buckets = 0;
  std::vector<int> atom_mol(natom, 0);
  for (int m = 0; m + 1 < (int)mol_atom_off.size(); ++m)
    for (int a = mol_atom_off[m]; a < mol_atom_off[m + 1]; ++a) atom_mol[a] = m;
  plan->max_mol_npoint = 0;
  for (int a = 0; a < natom; ++a) {
    const AtomLayout &L = *atoms[a];
    PoissonAtom &A = ha[a];
    const int n = L.nrad, lmax = lmax_of[a];
    if (n < 2) return set_error(kInvalidArgument, "radial grid needs >= 2 points");
    if (lmax < 0 || lmax > 20) return set_error(kNotSupported, "lmax must be in [0, 20]");
    const int lsize = (lmax + 1) * (lmax + 1);
    A.cx = L.center[0];
    A.cy = L.center[1];
    A.cz = L.center[2];
    A.first_x = L.r[0];
    A.last_x = L.r[n - 1];
    A.rt = L.rt;
    A.point_off = L.point_off;
    A.nrad = n;
    A.nang = L.nang;
    A.lmax = lmax;
    A.rad_off = (int)rad.size();
    rad.insert(rad.end(), L.r.begin(), L.r.end());
    rad.insert(rad.end(), L.wr.begin(), L.wr.end());
    rad.insert(rad.end(), L.j1.begin(), L.j1.end());
    rad.insert(rad.end(), L.j2.begin(), L.j2.end());
    rad.insert(rad.end(), L.j3.begin(), L.j3.end());
    rad.insert(rad.end(), L.sigma.begin(), L.sigma.end());
    // Thomas constants of the (2 1 / 1 4 1 / ... / 1 2) spline system
    std::vector<double> den(n), up(n, 0.0);
    den[0] = 2.0;
    up[0] = 1.0 / 2.0;
    for (int i = 1; i < n; ++i) {
      den[i] = ((i < n - 1) ? 4.0 : 2.0) - up[i - 1] * 1.0;
      if (i < n - 1) up[i] = 1.0 / den[i];
    }
    rad.insert(rad.end(), den.begin(), den.end());
    rad.insert(rad.end(), up.begin(), up.end());
    // one table per (angular rule, lmax); rules are identified by their
    // first direction and size, which is unique among Lebedev rules
    auto key = std::make_pair(L.nang, lmax);
    auto it = ykey.find(key);
    if (it == ykey.end()) {
      std::vector<double> y;
      ytable(L.ang, L.nang, lmax, y);
      ykey[key] = (int)ytab.size();
      A.ytab_off = (int)ytab.size();
      ytab.insert(ytab.end(), y.begin(), y.end());
    } else {
      A.ytab_off = it->second;
    }
    A.proj_off = (int)proj;
    proj += (long)n * lsize;
    A.spl_off = (int)spl;
    spl += (long)(n - 1) * lsize * 4;
    A.amp_off = (int)amp;
    amp += (long)lsize * 2;
    A.raw_off = (int)raw;
    raw += (long)lsize * n;
    A.scr_off = scr;
    scr += 3L * n * lsize;
    npts = std::max(npts, (long)L.point_off + (long)n * L.nang);
    A.sys_off = (int)sys_atom.size();
    const int mol = atom_mol[a];
    A.mol_point_start = mol_point_off[mol];
    A.mol_npoint = mol_point_off[mol + 1] - mol_point_off[mol];
    plan->max_mol_npoint = std::max(plan->max_mol_npoint, A.mol_npoint);
    A.bucket_off = buckets;
    buckets += n + 1;
    A.pair_off = pairs;
    pairs += A.mol_npoint;
    for (int l = 0; l <= lmax; ++l) {
      sys_atom.push_back(a);
      sys_l.push_back(l);
    }
    d.max_lmax = std::max(d.max_lmax, lmax);
    d.max_nrad = std::max(d.max_nrad, n);
    d.max_nang = std::max(d.max_nang, L.nang);
  }
  d.nsys = (int)sys_atom.size();
  NAPMO_TRY_CUDA(plan->atoms.upload(ha, s), "upload atoms");
  NAPMO_TRY_CUDA(plan->mol_atom_off.upload(mol_atom_off, s), "upload");
  NAPMO_TRY_CUDA(plan->mol_point_off.upload(mol_point_off, s), "upload");
  NAPMO_TRY_CUDA(plan->sys_atom.upload(sys_atom, s), "upload");
  NAPMO_TRY_CUDA(plan->sys_l.upload(sys_l, s), "upload");
  NAPMO_TRY_CUDA(plan->rad.upload(rad, s), "upload radial tables");
  NAPMO_TRY_CUDA(plan->ytab.upload(ytab, s), "upload harmonics");
  NAPMO_TRY_CUDA(plan->proj.alloc(proj), "alloc");
  NAPMO_TRY_CUDA(plan->spl.alloc(spl), "alloc");
  NAPMO_TRY_CUDA(plan->amp.alloc(amp), "alloc");
  NAPMO_TRY_CUDA(plan->raw_y.alloc(raw), "alloc");
  NAPMO_TRY_CUDA(plan->raw_dt.alloc(raw), "alloc");
  NAPMO_TRY_CUDA(plan->rscr.alloc(scr), "alloc");
  NAPMO_TRY_CUDA(plan->pg.alloc(npts), "alloc");
  d.atoms = plan->atoms.p;
  d.mol_atom_off = plan->mol_atom_off.p;
  d.mol_point_off = plan->mol_point_off.p;
  d.sys_atom = plan->sys_atom.p;
  d.sys_l = plan->sys_l.p;
  d.rad = plan->rad.p;
  d.ytab = plan->ytab.p;
  d.proj = plan->proj.p;
  d.spl = plan->spl.p;
  d.amp = plan->amp.p;
  d.raw_y = plan->raw_y.p;
  d.raw_dt = plan->raw_dt.p;
  d.rscr = plan->rscr.p;
  d.pg = plan->pg.p;
  d.npair = pairs;
  // LU factors of the radial systems (they depend on the grid only)
  d.lu_stride = 2 * d.max_nrad;
  NAPMO_TRY_CUDA(plan->lu.alloc((size_t)d.nsys * d.lu_stride * kW), "alloc radial LU");
  NAPMO_TRY_CUDA(plan->lmul.alloc((size_t)d.nsys * d.lu_stride * kKL), "alloc radial LU");
  NAPMO_TRY_CUDA(plan->lpiv.alloc((size_t)d.nsys * d.lu_stride), "alloc radial LU");
  d.lu = plan->lu.p;
  d.lmul = plan->lmul.p;
  d.lpiv = plan->lpiv.p;
  NAPMO_TRY_CUDA(launch_poisson_factor(d, s), "radial LU");
  return kOk;
}

// Pairs per evaluation item (CTA of chunk / 2 threads): a larger item shares
// one staging of its interval's coefficients among more pairs, but leaves
// fewer CTAs and, at 256 threads and 76 registers, fewer resident warps.  On B200,
// 512-pair items made the C20H42 100x302 evaluation 5 % faster (about 15,000
// pairs per interior bucket) and the H2O 50x110 and HCN 100x302 SCFs (300
// and 900 pairs) slower than 128-pair items.
static int eval_chunk_for(const std::vector<int> &count, const std::vector<PoissonAtom> &ha) {
  long pairs = 0, buckets = 0;
  for (const PoissonAtom &a : ha)
    for (int b = 1; b < a.nrad; ++b) {
      const int c = count[a.bucket_off + b];
      if (c > 0) {
        pairs += c;
        ++buckets;
      }
    }
  return buckets > 0 && pairs >= 4096L * buckets ? kEvalChunkMax : kEvalChunk;
}

// Bucket-sorted (atom, point) pair lists for the evaluation of the potential
// at the points (x, y, z) (device, all molecules concatenated), into pairs /
// items; with `keep` only the points whose flag is set.  Built once per grid
// (and once per screening mask); about 12 bytes per pair.  Synchronises `s`.
int build_pair_lists(PoissonPlan *plan, const double *x, const double *y, const double *z,
                     const int *keep, DevBuf<int> &pairs, DevBuf<double2> &pair_u,
                     DevBuf<EvalItem> &items, int &nitems, int &nitems_in, int &chunk,
                     cudaStream_t s) {
  PoissonDev &d = plan->d;
  const std::vector<PoissonAtom> &ha = plan->h_atoms;
  int nb = 0;
  for (auto &a : ha) nb += a.nrad + 1;
  DevBuf<int> bucket_of, count;
  NAPMO_TRY_CUDA(bucket_of.alloc(d.npair), "pair lists");
  NAPMO_TRY_CUDA(count.alloc(nb), "pair lists");
  NAPMO_TRY_CUDA(cudaMemsetAsync(count.p, 0, nb * sizeof(int), s), "pair lists");
  NAPMO_TRY_CUDA(launch_pair_buckets(d, plan->max_mol_npoint, x, y, z, keep, bucket_of.p,
                                     count.p, s),
                 "pair buckets");
  std::vector<int> hc(nb);
  NAPMO_TRY_CUDA(cudaMemcpyAsync(hc.data(), count.p, nb * sizeof(int), cudaMemcpyDeviceToHost, s),
                 "pair lists");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "pair lists");
  // exclusive scan per atom -> bucket starts (relative to the atom's slice)
  std::vector<int> start(nb);
  std::vector<EvalItem> hitems;
  chunk = eval_chunk_for(hc, ha);
  for (int a = 0; a < (int)ha.size(); ++a) {
    int acc = 0;
    for (int b = 0; b <= ha[a].nrad; ++b) {
      const int k = ha[a].bucket_off + b;
      start[k] = acc;
      for (int c = 0; c < hc[k]; c += chunk)
        hitems.push_back(EvalItem{a, b, acc + c, std::min(chunk, hc[k] - c)});
      acc += hc[k];
    }
  }
  NAPMO_TRY_CUDA(count.upload(start, s), "pair lists");  // reused as the cursor
  NAPMO_TRY_CUDA(pairs.alloc(d.npair), "pair lists");
  NAPMO_TRY_CUDA(pair_u.alloc(d.npair), "pair lists");
  d.pairs = pairs.p;
  d.pair_u = pair_u.p;
  NAPMO_TRY_CUDA(launch_pair_scatter(d, plan->max_mol_npoint, x, y, z, bucket_of.p, count.p, s),
                 "pair scatter");
  // interior buckets first, the tails after them: the evaluation runs them as
  // two kernels, each with the code of its own region only
  std::stable_partition(hitems.begin(), hitems.end(), [&](const EvalItem &it) {
    return it.bucket > 0 && it.bucket < ha[it.atom].nrad;
  });
  nitems_in = 0;
  for (const EvalItem &it : hitems) nitems_in += (it.bucket > 0 && it.bucket < ha[it.atom].nrad);
  NAPMO_TRY_CUDA(items.upload(hitems, s), "pair lists");
  if (!plan->pair_v.p) NAPMO_TRY_CUDA(plan->pair_v.alloc(d.npair), "pair lists");
  if (!plan->lcut.p) NAPMO_TRY_CUDA(plan->lcut.alloc(nb), "pair lists");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "pair lists");
  nitems = (int)hitems.size();
  d.pair_v = plan->pair_v.p;
  return kOk;
}

// Points the evaluation runs on: all (keep null) or the screened ones.
static int select_pair_lists(PoissonPlan *p, BeckeGrid *g, const int *keep,
                             unsigned long long key, cudaStream_t s) {
  PoissonDev &d = p->d;
  if (keep && key != p->screen_key) {
    p->screen_key = 0;
    const int st = build_pair_lists(p, g->dev.x, g->dev.y, g->dev.z, keep, p->pairs_s,
                                    p->pair_u_s, p->items_s, p->nitems_s, p->nitems_in_s,
                                    p->chunk_s, s);
    if (st) return st;
    p->screen_key = key;
  }
  d.keep = keep;
  d.pairs = keep ? p->pairs_s.p : p->pairs.p;
  d.pair_u = keep ? p->pair_u_s.p : p->pair_u.p;
  d.items = keep ? p->items_s.p : p->items.p;
  d.nitems = keep ? p->nitems_s : p->nitems;
  d.nitems_inner = keep ? p->nitems_in_s : p->nitems_in;
  d.eval_chunk = keep ? p->chunk_s : p->chunk;
  return kOk;
}

// Plan for one molecular grid, cached on the grid: a common lmax, or with
// lmax == kLmaxPerAtom each atom's own lebedev_precision(nang) / 2 (grids whose
// atoms carry different Lebedev rules).
int grid_poisson_plan(BeckeGrid *g, int lmax, cudaStream_t s, PoissonPlan **out) {
  if (g->layout.empty())
    return set_error(kNotSupported, "grid has no atomic structure (read from points)");
  if (g->poisson && g->poisson->lmax == lmax) {
    *out = g->poisson;
    return kOk;
  }
  delete g->poisson;
  g->poisson = nullptr;
  auto *p = new PoissonPlan;
  std::vector<const AtomLayout *> atoms;
  for (auto &L : g->layout) atoms.push_back(&L);
  std::vector<int> lm(atoms.size(), lmax);
  if (lmax == kLmaxPerAtom) {
    for (size_t a = 0; a < atoms.size(); ++a) {
      const int prec = lebedev_precision(atoms[a]->nang);
      if (prec < 0) {
        delete p;
        return set_error(kInvalidArgument, "no Lebedev rule with this number of points");
      }
      lm[a] = prec / 2;
    }
  } else if (lmax < 0) {
    delete p;
    return set_error(kInvalidArgument, "lmax must be >= 0 or kLmaxPerAtom");
  }
  int st = build_poisson_plan(atoms, lm, {0, (int)atoms.size()}, {0, g->size}, s, p);
  if (st != kOk) {
    delete p;
    return st;
  }
  st = build_pair_lists(p, g->dev.x, g->dev.y, g->dev.z, nullptr, p->pairs, p->pair_u,
                        p->items, p->nitems, p->nitems_in, p->chunk, s);
  if (st != kOk) {
    delete p;
    return st;
  }
  p->d.items = p->items.p;
  p->d.nitems = p->nitems;
  p->d.nitems_inner = p->nitems_in;
  p->d.eval_chunk = p->chunk;
  p->lmax = lmax;
  g->poisson = p;
  *out = p;
  return kOk;
}

// One Poisson solve on the grid's plan: v (=, += with accumulate) = V_H[rho].
// tol > 0 truncates the evaluation (see eval_tol); keep (grid flags, or null)
// restricts the evaluation to the flagged points, v = 0 elsewhere (its pair
// lists are built, synchronously, the first time a mask is used; key names
// the mask, which an address could not: a freed mask's address is reused).
// Several molecular grids as one, for Poisson solves of a batch in one launch
// per pipeline stage: the atoms of every grid in order, their points
// concatenated (grid m from off[m], no padding) in copies of the device
// arrays, and a Poisson plan with one molecule per grid, so that every atom
// pairs with its own molecule's points only.  lmax[m] is grid m's cutoff
// (kLmaxPerAtom: each atom's own rule).  The result owns its arrays and plan.
int grid_concat(const std::vector<BeckeGrid *> &grids, const std::vector<int> &lmax,
                cudaStream_t s, BeckeGrid **out, std::vector<int> *off) {
  std::unique_ptr<BeckeGrid> g(new BeckeGrid);
  std::vector<int> o(1, 0), mol_atom_off(1, 0), lm;
  for (size_t m = 0; m < grids.size(); ++m) {
    BeckeGrid *gm = grids[m];
    if (gm->layout.empty())
      return set_error(kNotSupported, "grid has no atomic structure (read from points)");
    for (const AtomLayout &L : gm->layout) {
      AtomLayout c = L;
      c.point_off += o.back();
      g->layout.push_back(c);
      int l = lmax[m];
      if (l == kLmaxPerAtom) {
        const int prec = lebedev_precision(L.nang);
        if (prec < 0) return set_error(kInvalidArgument, "no Lebedev rule with this number of points");
        l = prec / 2;
      }
      lm.push_back(l);
    }
    mol_atom_off.push_back((int)g->layout.size());
    o.push_back(o.back() + gm->size);
  }
  g->size = o.back();
  g->ncenter = (int)g->layout.size();
  DeviceGrid &d = g->dev;
  d.npoint = g->size;
  for (double **arr : {&d.x, &d.y, &d.z, &d.w, &d.wb})
    NAPMO_TRY_CUDA(cudaMalloc(arr, std::max(g->size, 1) * sizeof(double)), "alloc batch grid");
  for (size_t m = 0; m < grids.size(); ++m) {
    const DeviceGrid &src = grids[m]->dev;
    const size_t bytes = (size_t)grids[m]->size * sizeof(double);
    const long at = o[m];
    NAPMO_TRY_CUDA(cudaMemcpyAsync(d.x + at, src.x, bytes, cudaMemcpyDeviceToDevice, s), "copy");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(d.y + at, src.y, bytes, cudaMemcpyDeviceToDevice, s), "copy");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(d.z + at, src.z, bytes, cudaMemcpyDeviceToDevice, s), "copy");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(d.w + at, src.w, bytes, cudaMemcpyDeviceToDevice, s), "copy");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(d.wb + at, src.wb, bytes, cudaMemcpyDeviceToDevice, s), "copy");
  }
  auto *p = new PoissonPlan;
  g->poisson = p;  // owned by g from here on
  std::vector<const AtomLayout *> atoms;
  for (auto &L : g->layout) atoms.push_back(&L);
  int st = build_poisson_plan(atoms, lm, mol_atom_off, o, s, p);
  if (st != kOk) return st;
  st = build_pair_lists(p, d.x, d.y, d.z, nullptr, p->pairs, p->pair_u, p->items, p->nitems,
                        p->nitems_in, p->chunk, s);
  if (st != kOk) return st;
  p->d.items = p->items.p;
  p->d.nitems = p->nitems;
  p->d.nitems_inner = p->nitems_in;
  p->d.eval_chunk = p->chunk;
  p->lmax = -3;  // not a single-grid cutoff: grid_poisson_plan never reuses it
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "batch grid");
  *off = o;
  *out = g.release();
  return kOk;
}

void grid_free(BeckeGrid *g) { delete g; }

int run_poisson(BeckeGrid *g, PoissonPlan *p, const double *rho_dev, double *v_dev,
                bool accumulate, cudaStream_t s, double tol, const int *keep,
                unsigned long long key) {
  int st = select_pair_lists(p, g, keep, key, s);
  if (st) return st;
  p->d.eval_tol = tol;
  p->d.lcut = tol > 0.0 ? p->lcut.p : nullptr;
  NAPMO_TRY_CUDA(launch_poisson_project(p->d, rho_dev, g->dev.wb, g->dev.w, s), "project");
  NAPMO_TRY_CUDA(launch_poisson_radial(p->d, s), "radial solve");
  NAPMO_TRY_CUDA(launch_poisson_evaluate(p->d, g->size, g->dev.x, g->dev.y, g->dev.z,
                                         v_dev, accumulate, s),
                 "evaluate");
  return kOk;
}

// The grid's Poisson tables for `lmax`, set up for an operator evaluation:
// every point, no truncation, no raw spline output.
static int operator_dev(BeckeGrid *g, int lmax, cudaStream_t s, PoissonDev *out,
                        PoissonPlan **plan = nullptr) {
  PoissonPlan *p = nullptr;
  int st = grid_poisson_plan(g, lmax, s, &p);
  if (st) return st;
  if (plan) *plan = p;
  st = select_pair_lists(p, g, nullptr, 0, s);
  if (st) return st;
  *out = p->d;
  out->eval_tol = 0.0;
  out->lcut = nullptr;
  out->raw_y = nullptr;
  out->raw_dt = nullptr;
  return kOk;
}

// src = phi doi - resid (ndpsi.py:29)
__global__ void dpsi_source_kernel(int n, const double *__restrict__ phi,
                                   const double *__restrict__ resid, double doi,
                                   double *__restrict__ src) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) src[p] = phi[p] * doi - resid[p];
}

static cudaError_t launch_dpsi_source(int n, const double *phi, const double *resid, double doi,
                                      double *src, cudaStream_t s) {
  dpsi_source_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, phi, resid, doi, src);
  return cudaGetLastError();
}

// One CTA per (i, j): a fixed strided partition of the points and a fixed
// reduction tree, so every entry is reproducible.
__global__ void __launch_bounds__(256)
operator_matrix_kernel(int npoint, const double *__restrict__ A, long lda,
                       const double *__restrict__ B, long ldb, const double *__restrict__ wb,
                       const double *__restrict__ w, double *__restrict__ M, int m) {
  const int i = blockIdx.y, j = blockIdx.x;
  const double *a = A + (long)i * lda, *b = B + (long)j * ldb;
  double acc = 0.0;
  for (int p = threadIdx.x; p < npoint; p += 256) acc += a[p] * b[p] * wb[p] * w[p];
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) M[(long)i * m + j] = red[0];
}

static cudaError_t launch_operator_matrix(int npoint, int n, int m, const double *A, long lda,
                                          const double *B, long ldb, const double *wb,
                                          const double *w, double *M, cudaStream_t s) {
  if (n > 65535) return cudaErrorInvalidValue;
  operator_matrix_kernel<<<dim3(m, n), 256, 0, s>>>(npoint, A, lda, B, ldb, wb, w, M, m);
  return cudaGetLastError();
}

// k solves on the plan's grid (v[j] = V_H[rho[j]], rows ld apart): the
// projection, radial and evaluation launches each take a batch of solves, whose
// per-solve tables live in the plan's batch workspace (at most 512 MB; larger
// k runs in several batches).  Results equal k calls of run_poisson.
int run_poisson_many(BeckeGrid *g, PoissonPlan *p, int k, const double *rho_dev, long ld,
                     double *v_dev, cudaStream_t s, double tol, const int *keep,
                     unsigned long long key) {
  if (k <= 0) return kOk;
  int st = select_pair_lists(p, g, keep, key, s);
  if (st) return st;
  const PoissonDev &d = p->d;
  const size_t nd = p->proj.n + p->spl.n + p->amp.n + p->pair_v.n + p->rscr.n + p->pg.n;
  const size_t per = nd * sizeof(double) + p->lcut.n * sizeof(int);
  // grid limits: the projection and truncation launches use natom x B blocks
  // in y/z, the radial one B in y
  long B = std::min<long>(k, (long)((512ull << 20) / std::max<size_t>(per, 1)));
  B = std::min<long>(B, 65535 / std::max(d.natom, 1));
  if (B < 2 || !d.items) {
    for (int j = 0; j < k; ++j) {
      st = run_poisson(g, p, rho_dev + (long)j * ld, v_dev + (long)j * ld, false, s, tol, keep,
                       key);
      if (st) return st;
    }
    return kOk;
  }
  if (p->batch_ws.n < per * B) {
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "batch workspace");
    NAPMO_TRY_CUDA(p->batch_ws.alloc(per * B), "batch workspace");
  }
  PoissonDev P = d;
  P.batch_ld = ld;
  P.proj_stride = (long)p->proj.n;
  P.spl_stride = (long)p->spl.n;
  P.amp_stride = (long)p->amp.n;
  P.pairv_stride = (long)p->pair_v.n;
  P.lcut_stride = (long)p->lcut.n;
  P.rscr_stride = (long)p->rscr.n;
  double *ws = (double *)p->batch_ws.p;
  P.proj = ws;
  P.spl = P.proj + P.proj_stride * B;
  P.amp = P.spl + P.spl_stride * B;
  P.pair_v = P.amp + P.amp_stride * B;
  P.rscr = P.pair_v + P.pairv_stride * B;
  P.pg_stride = (long)p->pg.n;
  P.pg = P.rscr + P.rscr_stride * B;
  P.lcut = tol > 0.0 ? (int *)(P.pg + P.pg_stride * B) : nullptr;
  P.eval_tol = tol;
  P.raw_y = nullptr;
  P.raw_dt = nullptr;
  for (long j0 = 0; j0 < k; j0 += B) {
    P.nbatch = (int)std::min<long>(B, k - j0);
    NAPMO_TRY_CUDA(launch_poisson_project(P, rho_dev + j0 * ld, g->dev.wb, g->dev.w, s),
                   "project");
    NAPMO_TRY_CUDA(launch_poisson_radial(P, s), "radial solve");
    NAPMO_TRY_CUDA(launch_poisson_evaluate(P, g->size, g->dev.x, g->dev.y, g->dev.z,
                                           v_dev + j0 * ld, false, s),
                   "evaluate");
  }
  return kOk;
}

BeckeGrid::~BeckeGrid() {
  delete poisson;
  cudaFree(dev.x);
  cudaFree(dev.y);
  cudaFree(dev.z);
  cudaFree(dev.w);
  cudaFree(dev.wb);
  cudaFree(dev.origin);
  cudaFree(dev.radii);
  cudaFree(dev.atom_offset);
}

// Upload points (SoA), weights and centres.
static int upload_grid(BeckeGrid *g, cudaStream_t s) {
  const int n = g->size;
  std::vector<double> x(n), y(n), z(n);
  for (int i = 0; i < n; ++i) {
    x[i] = g->points[3 * i];
    y[i] = g->points[3 * i + 1];
    z[i] = g->points[3 * i + 2];
  }
  DevBuf<double> bx, by, bz, bw, bwb, bo, br;
  DevBuf<int> boff;
  NAPMO_TRY_CUDA(bx.upload(x, s), "upload grid");
  NAPMO_TRY_CUDA(by.upload(y, s), "upload grid");
  NAPMO_TRY_CUDA(bz.upload(z, s), "upload grid");
  NAPMO_TRY_CUDA(bw.upload(g->weights, s), "upload grid");
  NAPMO_TRY_CUDA(bwb.alloc(n), "alloc grid");
  NAPMO_TRY_CUDA(bo.upload(g->origin, s), "upload grid");
  NAPMO_TRY_CUDA(br.upload(g->radii, s), "upload grid");
  NAPMO_TRY_CUDA(boff.upload(g->atom_offset, s), "upload grid");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "upload grid");
  g->dev.npoint = n;
  g->dev.ncenter = g->ncenter;
  g->dev.x = bx.release();
  g->dev.y = by.release();
  g->dev.z = bz.release();
  g->dev.w = bw.release();
  g->dev.wb = bwb.release();
  g->dev.origin = bo.release();
  g->dev.radii = br.release();
  g->dev.atom_offset = boff.release();
  return kOk;
}

static double distance_ref(const double *a, const double *b) {
  double out = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double d = a[i] - b[i];
    out += d * d;
  }
  return sqrt(out);
}

// Becke weights of a grid on the device; tables R_ij / a_ij built on the host
// exactly as nAPMO does (src/grid/becke.cpp:80-115).
int compute_becke(BeckeGrid *g, cudaStream_t s) {
  const int nc = g->ncenter;
  const int tri = nc * (nc + 1) / 2;
  std::vector<double> R(tri), A(tri);
  int off = 0;
  for (int i = 0; i < nc; ++i)
    for (int j = 0; j <= i; ++j) R[off++] = distance_ref(&g->origin[3 * i], &g->origin[3 * j]);
  off = 0;
  for (int i = 0; i < nc; ++i)
    for (int j = 0; j <= i; ++j) {
      double aux = (g->radii[i] - g->radii[j]) / (g->radii[i] + g->radii[j]);
      aux = aux / (aux * aux - 1.0);
      if (aux > 0.45) aux = 0.45;
      else if (aux < -0.45) aux = -0.45;
      A[off++] = aux;
    }
  DevBuf<double> dR, dA;
  NAPMO_TRY_CUDA(dR.upload(R, s), "becke tables");
  NAPMO_TRY_CUDA(dA.upload(A, s), "becke tables");
  cudaError_t e = launch_becke_weights(g->size, nc, g->dev.x, g->dev.y, g->dev.z,
                                       g->dev.origin, dR.p, dA.p, g->dev.atom_offset,
                                       g->dev.wb, s);
  if (e == cudaErrorInvalidValue)
    return set_error(kNotSupported, "Becke weights: too many centres for one grid");
  NAPMO_TRY_CUDA(e, "becke kernel");
  g->becke_weights.resize(g->size);
  NAPMO_TRY_CUDA(cudaMemcpyAsync(g->becke_weights.data(), g->dev.wb,
                                 g->size * sizeof(double), cudaMemcpyDeviceToHost, s),
                 "becke download");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "becke sync");
  return kOk;
}

// ------------------------------------------------- generic decomposition
// Per-spline extrapolation for the generic evaluation entry point.
struct SplineDesc {
  int left_kind, right_kind;  // 0 zero, 1 cusp exp, 2 power-law, 3 potential
  double l0, l1, l2;          // left: cusp a0,b0,x0 | potential amp_left, l
  double r0, r1;              // right: power amp, power | potential amp, l
  int n;
  int off;                    // offset into y/dt arrays
};

__device__ double spline_eval_generic(const SplineDesc &sd, const RTParams &rt,
                                      double first_x, double last_x,
                                      const double *y, const double *dt, double x) {
  if (x < first_x) {
    switch (sd.left_kind) {
      case 1: return sd.l0 * exp(sd.l1 * (x - sd.l2));
      case 3: return sd.l0 * pow(x, sd.l1);
      default: return 0.0;
    }
  }
  if (x > last_x) {
    switch (sd.right_kind) {
      case 2: return sd.r0 * pow(x, sd.r1);
      case 3: return sd.r0 / pow(x, sd.r1 + 1);
      default: return 0.0;
    }
  }
  double t;
  switch (rt.kind) {
    case kRTChebyshev: t = -(acos((x - rt.p0) / (x + rt.p0)) / rt.p1) + rt.npoint; break;
    case kRTPower: t = pow(x / rt.p0, 1.0 / rt.p1) - 1; break;
    case kRTLinear: t = (x - rt.p0) / rt.p1; break;
    case kRTExp: t = log(x / rt.p0) / rt.p1; break;
    case kRTShiftedExp: t = log((x + rt.p1) / rt.p0) / rt.p2; break;
    default: t = x;
  }
  int j = (int)floor(t);
  if (j == sd.n - 1) j = sd.n - 2;
  if (j < 0) j = 0;
  const double u = t - j;
  const double *yy = y + sd.off, *dd = dt + sd.off;
  const double z = yy[j + 1] - yy[j];
  return yy[j] + u * (dd[j] + u * (3 * z - 2 * dd[j] - dd[j + 1] +
                                   u * (-2 * z + dd[j] + dd[j + 1])));
}

__global__ void decomposition_generic_kernel(int npoint, const double *__restrict__ pts,
                                             double cx, double cy, double cz,
                                             const SplineDesc *__restrict__ sds,
                                             int nspline, int lmax, RTParams rt,
                                             double first_x, double last_x, int has_tail,
                                             const double *__restrict__ y,
                                             const double *__restrict__ dt,
                                             double *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  const double dx = pts[3 * p] - cx, dy = pts[3 * p + 1] - cy, dz = pts[3 * p + 2] - cz;
  const double d = sqrt(dx * dx + dy * dy + dz * dz);
  if (!(d < last_x || has_tail)) return;
  const double inv_sqrt_4pi = 0.28209479177387814347;
  double acc = out[p];
  acc += spline_eval_generic(sds[0], rt, first_x, last_x, y, dt, d) * inv_sqrt_4pi;
  if (lmax > 0) {
    double work[(kMaxLmax + 1) * (kMaxLmax + 1)];
    work[0] = dz;
    work[1] = dx;
    work[2] = dy;
    if (lmax > 1) solid_harmonics(work, lmax);
    int counter = 0;
    double dpowl = 1.0;
    for (int l = 1; l <= lmax; ++l) {
      dpowl = dpowl / d;
      const double factor = sqrt((double)(2 * l + 1));
      for (int m = -l; m <= l; ++m) {
        const double s = spline_eval_generic(sds[counter + 1], rt, first_x, last_x, y, dt, d);
        acc += s * factor * inv_sqrt_4pi * dpowl * work[counter];
        counter++;
      }
    }
  }
  out[p] = acc;
}

// Moments of a segmented grid function (dot_multi_moments): pass 1 builds the
// per-point polynomial table, pass 2 sums each (segment, moment) in point order.
__global__ void moments_poly_kernel(long npoint, long nvector, const double *data,
                                    const double *pts, double cx, double cy, double cz,
                                    long lmax, long mtype, long nmoment, double *poly) {
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  double term = data[(nvector - 1) * npoint + p];
  for (long v = nvector - 2; v >= 0; v--) term *= data[v * npoint + p];
  double *row = poly + p * nmoment;
  row[0] = term;
  if (lmax > 0 && nmoment > 1) {
    const double d0 = pts[3 * p] - cx, d1 = pts[3 * p + 1] - cy, d2 = pts[3 * p + 2] - cz;
    double work[(kMaxLmax + 1) * (kMaxLmax + 1)];
    if (mtype == 1) {
      work[0] = d0; work[1] = d1; work[2] = d2;
      int old_off = 0, old_n = 3;
      for (int l = 2; l <= lmax; l++) {
        const int nn = old_n + l + 1, no = old_off + old_n;
        for (int i = 0; i < old_n; i++) work[no + i] = work[0] * work[old_off + i];
        for (int i = 0; i < l; i++) work[no + old_n + i] = work[1] * work[no - l + i];
        work[no + nn - 1] = work[2] * work[no - 1];
        old_n = nn;
        old_off = no;
      }
    } else if (mtype == 2) {
      work[0] = d2; work[1] = d0; work[2] = d1;
      solid_harmonics(work, lmax);
    } else if (mtype == 3) {
      work[0] = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
      for (long c = 0; c + 1 < lmax; ++c) work[c + 1] = work[0] * work[c];
    } else {
      const double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
      work[0] = d2 / r; work[1] = d0 / r; work[2] = d1 / r;
      solid_harmonics(work, lmax);
    }
    for (long i = 1; i < nmoment; ++i) row[i] = term * work[i - 1];
  }
}

__global__ void moments_sum_kernel(long nseg, const long *seg_begin, long nmoment,
                                   const double *poly, double *out) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= nseg * nmoment) return;
  const long s = e / nmoment, m = e % nmoment;
  double acc = out[e];
  for (long p = seg_begin[s]; p < seg_begin[s + 1]; ++p) acc += poly[p * nmoment + m];
  out[e] = acc;
}

// Deterministic sum of f * wb * w over a grid (two passes, fixed order).
__global__ void integrate_partial_kernel(int n, const double *f, const double *wb,
                                         const double *w, double *part) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc += f[i] * wb[i] * w[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void integrate_final_kernel(int nb, const double *part, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < nb; ++i) s += part[i];
    *out = s;
  }
}

int grid_integrate_dev(const BeckeGrid *g, const double *f_dev, double *out_dev,
                       cudaStream_t s) {
  const int nb = 148 * 2;
  DevBuf<double> part;
  NAPMO_TRY_CUDA(part.alloc(nb), "integrate");
  integrate_partial_kernel<<<nb, 256, 0, s>>>(g->size, f_dev, g->dev.wb, g->dev.w, part.p);
  integrate_final_kernel<<<1, 32, 0, s>>>(nb, part.p, out_dev);
  NAPMO_TRY_CUDA(cudaGetLastError(), "integrate");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "integrate");
  return kOk;
}

}  // namespace napmo

using namespace napmo;

template <class T, class F>
static T *make_or_null(F &&f) {
  T *out = nullptr;
  guarded([&] {
    out = f();
    return kOk;
  });
  return out;
}

// ======================================================================
extern "C" {

int napmo_last_error(char *buf, int len) { return last_error(buf, len); }

void napmo_free_array(double *p) { delete[] p; }

// -------------------------------------------------------------- transforms
void RTransform_del(RTransform *rt) { delete rt; }
double RTransform_radius(RTransform *rt, double t) { return rt->radius(t); }
double RTransform_deriv(RTransform *rt, double t) { return rt->deriv(t); }
double RTransform_deriv2(RTransform *rt, double t) { return rt->deriv2(t); }
double RTransform_deriv3(RTransform *rt, double t) { return rt->deriv3(t); }
double RTransform_inv(RTransform *rt, double r) { return rt->inv(r); }
void RTransform_radius_array(RTransform *rt, double *t, double *r, int n) {
  for (int i = 0; i < n; ++i) r[i] = rt->radius(t[i]);
}
void RTransform_deriv_array(RTransform *rt, double *t, double *d, int n) {
  for (int i = 0; i < n; ++i) d[i] = rt->deriv(t[i]);
}
void RTransform_deriv2_array(RTransform *rt, double *t, double *d, int n) {
  for (int i = 0; i < n; ++i) d[i] = rt->deriv2(t[i]);
}
void RTransform_deriv3_array(RTransform *rt, double *t, double *d, int n) {
  for (int i = 0; i < n; ++i) d[i] = rt->deriv3(t[i]);
}
void RTransform_inv_array(RTransform *rt, double *r, double *t, int n) {
  for (int i = 0; i < n; ++i) t[i] = rt->inv(r[i]);
}
int RTransform_get_npoint(RTransform *rt) { return rt->npoint; }

RTransform *IdentityRTransform_new(int n) {
  return make_or_null<RTransform>([&] {
    if (n < 2) throw std::domain_error("A radial grid consists of at least two points.");
    return new IdentityRT(n);
  });
}
RTransform *LinearRTransform_new(double a, double b, int n) {
  return make_or_null<RTransform>([&] { return new LinearRT(a, b, n); });
}
double LinearRTransform_get_rmin(LinearRT *r) { return r->rmin; }
double LinearRTransform_get_rmax(LinearRT *r) { return r->rmax; }
double LinearRTransform_get_alpha(LinearRT *r) { return r->alpha; }
RTransform *ExpRTransform_new(double a, double b, int n) {
  return make_or_null<RTransform>([&] { return new ExpRT(a, b, n); });
}
double ExpRTransform_get_rmin(ExpRT *r) { return r->rmin; }
double ExpRTransform_get_rmax(ExpRT *r) { return r->rmax; }
double ExpRTransform_get_alpha(ExpRT *r) { return r->alpha; }
RTransform *ShiftedExpRTransform_new(double a, double s, double b, int n) {
  return make_or_null<RTransform>([&] { return new ShiftedExpRT(a, s, b, n); });
}
double ShiftedExpRTransform_get_rmin(ShiftedExpRT *r) { return r->rmin; }
double ShiftedExpRTransform_get_rshift(ShiftedExpRT *r) { return r->rshift; }
double ShiftedExpRTransform_get_rmax(ShiftedExpRT *r) { return r->rmax; }
double ShiftedExpRTransform_get_r0(ShiftedExpRT *r) { return r->r0; }
double ShiftedExpRTransform_get_alpha(ShiftedExpRT *r) { return r->alpha; }
RTransform *PowerRTransform_new(double a, double b, int n) {
  return make_or_null<RTransform>([&] { return new PowerRT(a, b, n); });
}
double PowerRTransform_get_rmin(PowerRT *r) { return r->rmin; }
double PowerRTransform_get_rmax(PowerRT *r) { return r->rmax; }
double PowerRTransform_get_power(PowerRT *r) { return r->power; }
RTransform *ChebyshevRTransform_new(double radii, int n) {
  return make_or_null<RTransform>([&] {
    if (n < 2) throw std::domain_error("A radial grid consists of at least two points.");
    return new ChebyshevRT(radii, n);
  });
}
double ChebyshevRTransform_get_radii(ChebyshevRT *r) { return r->radii; }
double ChebyshevRTransform_get_z(ChebyshevRT *r) { return r->z; }

// ------------------------------------------------------------ angular grid
AngularGrid *AngularGrid_new(int lorder) {
  return make_or_null<AngularGrid>([&] { return new AngularGrid(lorder); });
}
void AngularGrid_del(AngularGrid *g) { delete g; }
int AngularGrid_get_lorder(AngularGrid *g) { return g->lorder; }
double *AngularGrid_get_points(AngularGrid *g) { return g->points.data(); }
double *AngularGrid_get_weights(AngularGrid *g) { return g->weights.data(); }
// Points to (1, theta, phi) (src/grid/angular.cpp:39-50).
void AngularGrid_spherical(AngularGrid *g) {
  for (int i = 0; i < g->lorder; ++i) {
    double *q = &g->points[3 * i];
    const double x = q[0], y = q[1], z = q[2];
    const double t = acos(z);
    const double fact = sqrt(x * x + y * y);
    double ph = (0 < fact) ? acos(x / fact) : acos(x);
    if (y < 0) ph = -ph;
    q[0] = 1.0;
    q[1] = t;
    q[2] = ph;
  }
}
// 4 pi sum_j w_j s_j prod_seg f_seg(j) (src/grid/angular.cpp:142-163); a null
// `s` means s_j = 1.
double AngularGrid_integrate(AngularGrid *g, int segments, double *f, double *s) {
  double out = 0.0;
  for (int j = 0; j < g->lorder; ++j) {
    double v = f[j];
    for (int k = 1; k < segments; ++k) v *= f[k * g->lorder + j];
    out += s ? v * g->weights[j] * s[j] : v * g->weights[j];
  }
  return out * 4.0 * M_PI;
}
void AngularGrid_spherical_expansion(AngularGrid *, int, int, double *, double *) {
  set_error(kNotSupported,
            "AngularGrid.spherical_expansion (GSL spherical harmonics) is not part "
            "of the grid-quadrature path; use AtomicGrid.spherical_expansion");
}
void AngularGrid_eval_expansion(AngularGrid *, int, int, double *, double *) {
  set_error(kNotSupported,
            "AngularGrid.eval_expansion (GSL spherical harmonics) is not part of "
            "the grid-quadrature path");
}

// ------------------------------------------------------------- radial grid
RadialGrid *RadialGrid_new(RTransform *rtf, double rad) {
  return make_or_null<RadialGrid>([&] { return new RadialGrid(rtf, rad); });
}
void RadialGrid_del(RadialGrid *g) { delete g; }
double RadialGrid_integrate(RadialGrid *g, int segments, double *f) {
  return g->integrate(segments, f);
}
// (1/r) d^2/dr^2 (r f) at the grid's points (radial.cpp:51-192); returns a
// new[] array of size() values released by napmo_free_array.
double *RadialGrid_deriv2(RadialGrid *g, double *f) {
  return make_or_null<double>([&] {
    const int n = (int)g->points.size();
    std::unique_ptr<double[]> out(new double[n]);
    radial_deriv2(g->points.data(), n, g->radii, f, out.get());
    return out.release();
  });
}
int RadialGrid_get_size(RadialGrid *g) { return (int)g->points.size(); }
double RadialGrid_get_radii(RadialGrid *g) { return g->radii; }
double *RadialGrid_get_points(RadialGrid *g) { return g->points.data(); }
double *RadialGrid_get_weights(RadialGrid *g) { return g->weights.data(); }

// ------------------------------------------------------------- atomic grid
AtomicGrid *AtomicGrid_new(AngularGrid *a, RadialGrid *r, double *R) {
  return make_or_null<AtomicGrid>([&] { return new AtomicGrid(a, r, R); });
}
void AtomicGrid_del(AtomicGrid *g) { delete g; }
int AtomicGrid_get_size(AtomicGrid *g) { return g->size; }
double AtomicGrid_get_radii(AtomicGrid *g) { return g->radii; }
double *AtomicGrid_get_origin(AtomicGrid *g) { return g->origin; }
double *AtomicGrid_get_points(AtomicGrid *g) { return g->points.data(); }
double *AtomicGrid_get_weights(AtomicGrid *g) { return g->weights.data(); }

// Sum over `segments` blocks of `size` points of prod_f f (src/grid/
// atomic_grid.cpp:53-80).  Returns a new[] array released by napmo_free_array.
double *AtomicGrid_integrate(AtomicGrid *, int nfunc, int segments, int size, double *f) {
  const long total = (long)size * segments;
  double *out = new double[segments]();
  for (int i = 0; i < segments; ++i) {
    for (int j = 0; j < size; ++j) {
      const long k = (long)i * size + j;
      double v = f[k];
      for (int s = 1; s < nfunc; ++s) v *= f[s * total + k];
      out[i] += v;
    }
  }
  return out;
}

static AtomLayout layout_of(const AtomicGrid *ag, int point_off) {
  AtomLayout L;
  const RadialGrid *rg = ag->rad;
  const RTransform *rt = rg->rtf;
  L.rt = rt->params();
  L.nrad = (int)rg->points.size();
  L.nang = ag->ang->lorder;
  L.point_off = point_off;
  for (int d = 0; d < 3; ++d) L.center[d] = ag->origin[d];
  L.r = rg->points;
  L.wr = rg->weights;
  L.j1.resize(L.nrad);
  L.j2.resize(L.nrad);
  L.j3.resize(L.nrad);
  L.sigma.assign(L.nrad, 0.0);
  for (int i = 0; i < L.nrad; ++i) {
    const double t = i;
    L.j1[i] = rt->deriv(t);
    L.j2[i] = rt->deriv2(t);
    L.j3[i] = rt->deriv3(t);
    for (int j = 0; j < L.nang; ++j) L.sigma[i] += ag->weights[(size_t)i * L.nang + j];
  }
  L.ang = ag->ang->points;
  return L;
}

// Spherical expansion of f on one atomic grid (GPU projection kernel); returns
// new double[nrad * lsize] in [nrad][lsize] order, released by napmo_free_array.
double *AtomicGrid_spherical_expansion(AtomicGrid *ag, double *f, int lmax) {
  double *result = nullptr;
  guarded([&] {
    if (lmax < 0) return set_error(kInvalidArgument, "lmax can not be negative.");
    cudaStream_t s = host_api_stream();
    AtomLayout L = layout_of(ag, 0);
    PoissonPlan plan;
    int st = build_poisson_plan({&L}, {lmax}, {0, 1}, {0, ag->size}, s, &plan);
    if (st) return st;
    DevBuf<double> df, dw, dones;
    std::vector<double> ones(ag->size, 1.0);
    NAPMO_TRY_CUDA(df.upload(f, ag->size, s), "expansion");
    NAPMO_TRY_CUDA(dw.upload(ag->weights, s), "expansion");
    NAPMO_TRY_CUDA(dones.upload(ones, s), "expansion");
    NAPMO_TRY_CUDA(launch_poisson_project(plan.d, df.p, dones.p, dw.p, s), "expansion");
    const int lsize = (lmax + 1) * (lmax + 1);
    result = new double[(size_t)L.nrad * lsize];
    NAPMO_TRY_CUDA(cudaMemcpyAsync(result, plan.proj.p, (size_t)L.nrad * lsize * sizeof(double),
                                   cudaMemcpyDeviceToHost, s),
                   "expansion");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "expansion");
    return kOk;
  });
  return result;
}

// -------------------------------------------------------------- Becke grid
BeckeGrid *BeckeGrid_new(AtomicGrid **grids, int n, int l, double ld) {
  BeckeGrid *g = nullptr;
  int st = guarded([&] {
    g = new BeckeGrid;
    g->ncenter = n;
    g->ablmax = l;
    g->abldep = ld;
    g->atom_offset.push_back(0);
    for (int i = 0; i < n; ++i) {
      g->size += grids[i]->size;
      g->atom_offset.push_back(g->size);
    }
    g->radii.resize(n);
    g->origin.resize(3 * n);
    g->points.reserve(3 * (size_t)g->size);
    g->weights.reserve(g->size);
    for (int i = 0; i < n; ++i) {
      const AtomicGrid *ag = grids[i];
      g->atgrid.push_back(*ag);
      for (int d = 0; d < 3; ++d) g->origin[3 * i + d] = ag->origin[d];
      g->radii[i] = ag->radii;
      g->points.insert(g->points.end(), ag->points.begin(), ag->points.end());
      g->weights.insert(g->weights.end(), ag->weights.begin(), ag->weights.end());
      g->layout.push_back(layout_of(ag, g->atom_offset[i]));
    }
    cudaStream_t s = host_api_stream();
    int e = upload_grid(g, s);
    if (e) return e;
    return compute_becke(g, s);
  });
  if (st != kOk) {
    delete g;
    return nullptr;
  }
  return g;
}

// Lowdin-compatible grid: p[size][4] = (x, y, z, becke weight), unit weights.
BeckeGrid *BeckeGrid_from_points(double *p, int sz, int nc) {
  BeckeGrid *g = nullptr;
  int st = guarded([&] {
    g = new BeckeGrid;
    g->size = sz;
    g->ncenter = nc;
    g->abldep = 1.0e-6;
    g->ablmax = 1;
    g->points.resize(3 * (size_t)sz);
    g->weights.assign(sz, 1.0);
    g->becke_weights.resize(sz);
    for (int i = 0; i < sz; ++i) {
      for (int d = 0; d < 3; ++d) g->points[3 * i + d] = p[4 * i + d];
      g->becke_weights[i] = p[4 * i + 3];
    }
    g->radii.assign(nc, 0.0);
    g->origin.assign(3 * (size_t)nc, 0.0);
    g->atom_offset.assign(nc + 1, sz);
    g->atom_offset[0] = 0;
    cudaStream_t s = host_api_stream();
    int e = upload_grid(g, s);
    if (e) return e;
    NAPMO_TRY_CUDA(cudaMemcpy(g->dev.wb, g->becke_weights.data(), sz * sizeof(double),
                              cudaMemcpyHostToDevice),
                   "upload becke weights");
    return kOk;
  });
  if (st != kOk) {
    delete g;
    return nullptr;
  }
  return g;
}

void BeckeGrid_del(BeckeGrid *g) { delete g; }
int BeckeGrid_get_ncenter(BeckeGrid *g) { return g->ncenter; }
int BeckeGrid_get_size(BeckeGrid *g) { return g->size; }
double *BeckeGrid_get_radii(BeckeGrid *g) { return g->radii.data(); }
double *BeckeGrid_get_points(BeckeGrid *g) { return g->points.data(); }
double *BeckeGrid_get_weights(BeckeGrid *g) { return g->weights.data(); }
double *BeckeGrid_get_origin(BeckeGrid *g) { return g->origin.data(); }
double *BeckeGrid_get_becke_weights(BeckeGrid *g) { return g->becke_weights.data(); }

double BeckeGrid_integrate(BeckeGrid *g, double *f) {
  double out = NAN;
  guarded([&] {
    cudaStream_t s = host_api_stream();
    DevBuf<double> df, dout;
    NAPMO_TRY_CUDA(df.upload(f, g->size, s), "integrate");
    NAPMO_TRY_CUDA(dout.alloc(1), "integrate");
    int st = grid_integrate_dev(g, df.p, dout.p, s);
    if (st) return st;
    NAPMO_TRY_CUDA(cudaMemcpy(&out, dout.p, sizeof(double), cudaMemcpyDeviceToHost), "integrate");
    return kOk;
  });
  return out;
}

// Moves the grid's centres to origin [ncenter][3] (bohr).  Each atomic grid's
// points are rebuilt around its new centre with the expression of its
// construction (atomic_grid.cpp:12-51, origin + r u), so the result equals a
// grid built at the new geometry bit for bit; the device mirror is rewritten
// in place (no allocation), the Becke weights recomputed and the Poisson
// tables dropped (rebuilt on next use).  The quadrature weights do not depend
// on the positions.  No counterpart in nAPMO, which builds a new grid per
// geometry.  Synchronises the library's host stream.
int napmo_grid_set_centers(BeckeGrid *g, const double *origin) {
  return guarded([&] {
    NAPMO_REQUIRE(!g->layout.empty() && (int)g->layout.size() == g->ncenter,
                  "grid has no atomic structure (read from points)");
    const int n = g->size;
    std::vector<double> x(n), y(n), z(n);
    for (int a = 0; a < g->ncenter; ++a) {
      AtomLayout &L = g->layout[a];
      AtomicGrid &ag = g->atgrid[a];
      for (int d = 0; d < 3; ++d) {
        g->origin[3 * a + d] = origin[3 * a + d];
        L.center[d] = origin[3 * a + d];
        ag.origin[d] = origin[3 * a + d];
      }
      for (int i = 0; i < L.nrad; ++i) {
        const double rp = L.r[i];
        for (int j = 0; j < L.nang; ++j) {
          const int k = i * L.nang + j;
          for (int d = 0; d < 3; ++d) ag.points[3 * k + d] = L.ang[3 * j + d] * rp + ag.origin[d];
          const long q = (long)L.point_off + k;
          for (int d = 0; d < 3; ++d) g->points[3 * q + d] = ag.points[3 * k + d];
          x[q] = ag.points[3 * k];
          y[q] = ag.points[3 * k + 1];
          z[q] = ag.points[3 * k + 2];
        }
      }
    }
    cudaStream_t s = host_api_stream();
    NAPMO_TRY_CUDA(cudaMemcpyAsync(g->dev.x, x.data(), n * sizeof(double), cudaMemcpyHostToDevice, s),
                   "move grid");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(g->dev.y, y.data(), n * sizeof(double), cudaMemcpyHostToDevice, s),
                   "move grid");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(g->dev.z, z.data(), n * sizeof(double), cudaMemcpyHostToDevice, s),
                   "move grid");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(g->dev.origin, g->origin.data(), g->origin.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, s),
                   "move grid");
    if (g->poisson) {
      NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "move grid");
      delete g->poisson;
      g->poisson = nullptr;
    }
    ++g->generation;
    return compute_becke(g, s);  // synchronises s before the host vectors go
  });
}

// Device pointers of the grid mirror: x, y, z, w, wb (each size long).
int napmo_grid_device_arrays(BeckeGrid *g, double **x, double **y, double **z,
                             double **w, double **wb) {
  *x = g->dev.x;
  *y = g->dev.y;
  *z = g->dev.z;
  *w = g->dev.w;
  *wb = g->dev.wb;
  return kOk;
}

// ------------------------------------------------------------------- Cell
// Only the non-periodic cell (nvec = 0) is meaningful on molecular grids.
void *Cell_new(double *, int nvec) {
  if (nvec != 0) {
    set_error(kNotSupported, "periodic cells are not used by molecular grids");
    return nullptr;
  }
  return new int(0);
}
void Cell_del(void *c) { delete static_cast<int *>(c); }

// ----------------------------------------------------------- cubic spline
void solve_cubic_spline_system(double *y, double *dt, int npoint) {
  cubic_spline_dt(y, dt, npoint);
}
void tridiagsym_solve(double *mid, double *up, double *right, double *sol, int n) {
  tridiag_sym_solve(mid, up, right, sol, n);
}
// Integration weights of a cubic spline on the uniform t-axis.
void compute_cubic_spline_int_weights(double *weights, int npoint) {
  std::vector<double> y(npoint, 0.0), dt(npoint);
  for (int i = 0; i < npoint; ++i) {
    if (i > 0) y[i - 1] = 0.0;
    y[i] = 1.0;
    cubic_spline_dt(y.data(), dt.data(), npoint);
    double w = y[i];
    if (i == 0 || i == npoint - 1) w *= 0.5;
    w += (dt[0] - dt[npoint - 1]) / 12.0;
    weights[i] = w;
  }
}
CubicSpline *CubicSpline_new(double *y, double *dt, Extrapolation *e, RTransform *r, int n) {
  return make_or_null<CubicSpline>([&] { return new CubicSpline(y, dt, e, r, n); });
}
void CubicSpline_del(CubicSpline *c) { delete c; }
void CubicSpline_eval(CubicSpline *c, double *x, double *y, int n) {
  for (int i = 0; i < n; ++i) y[i] = c->eval(x[i]);
}
void CubicSpline_eval_deriv(CubicSpline *c, double *x, double *d, int n) {
  for (int i = 0; i < n; ++i) d[i] = c->eval_deriv(x[i]);
}
double CubicSpline_get_first_x(CubicSpline *c) { return c->first_x; }
double CubicSpline_get_last_x(CubicSpline *c) { return c->last_x; }
RTransform *CubicSpline_get_rtransform(CubicSpline *c) { return c->rtf; }
Extrapolation *CubicSpline_get_extrapolation(CubicSpline *c) { return c->ext; }

void Extrapolation_prepare(Extrapolation *e, CubicSpline *c) { e->prepare(c); }
void Extrapolation_del(Extrapolation *e) { delete e; }
double Extrapolation_eval_left(Extrapolation *e, double x) { return e->eval_left(x); }
double Extrapolation_eval_right(Extrapolation *e, double x) { return e->eval_right(x); }
double Extrapolation_deriv_left(Extrapolation *e, double x) { return e->deriv_left(x); }
double Extrapolation_deriv_right(Extrapolation *e, double x) { return e->deriv_right(x); }
bool Extrapolation_has_tail(Extrapolation *e) { return e->has_tail(); }
Extrapolation *ZeroExtrapolation_new() { return new ZeroExtrapolation(); }
Extrapolation *CuspExtrapolation_new() { return new CuspExtrapolation(); }
Extrapolation *PowerExtrapolation_new(double p) { return new PowerExtrapolation(p); }
double PowerExtrapolation_get_power(PowerExtrapolation *e) { return e->power; }
Extrapolation *PotentialExtrapolation_new(int l) {
  return make_or_null<Extrapolation>([&] {
    if (l < 0) throw std::domain_error("The argument l cannot be negative.");
    return new PotentialExtrapolation(l);
  });
}

// ------------------------------------------------------------ ODE (host)
void build_ode2(double *b, double *a, double *f, double *bcs, double *coeffs,
                double *rhs, long npoint) {
  build_ode2_matrix(b, a, f, bcs, coeffs, rhs, npoint);
}
double hermite_overlap2(long xmax, long i0, bool d0, long i1, bool d1) {
  return napmo::hermite_overlap2(xmax, i0, d0, i1, d1);
}
double hermite_overlap3(long xmax, long i0, bool d0, long i1, bool d1, long i2, bool d2) {
  return napmo::hermite_overlap3(xmax, i0, d0, i1, d1, i2, d2);
}
void fill_pure_polynomials(double *out, long lmax) { solid_harmonics(out, lmax); }

// ------------------------------------------- decomposition / moments (GPU)
void eval_decomposition_grid(CubicSpline **splines, double *center, double *output,
                             double *points, void *cell, long nspline, long npoint) {
  guarded([&] {
    (void)cell;
    const long lmax = (long)std::sqrt((double)nspline) - 1;
    if ((lmax + 1) * (lmax + 1) != nspline)
      return set_error(kInvalidArgument,
                       "The number of splines does not match a well-defined lmax.");
    if (lmax > kMaxLmax) return set_error(kNotSupported, "lmax too large");
    std::vector<SplineDesc> sd(nspline);
    std::vector<double> y, dt;
    for (long i = 0; i < nspline; ++i) {
      CubicSpline *c = splines[i];
      SplineDesc &d = sd[i];
      d = SplineDesc();
      d.n = c->n;
      d.off = (int)y.size();
      y.insert(y.end(), c->y, c->y + c->n);
      dt.insert(dt.end(), c->dt, c->dt + c->n);
      if (auto *p = dynamic_cast<PotentialExtrapolation *>(c->ext)) {
        d.left_kind = 3;
        d.l0 = p->amp_left;
        d.l1 = (double)p->l;
        d.right_kind = 3;
        d.r0 = p->amp_right;
        d.r1 = (double)p->l;
      } else if (auto *q = dynamic_cast<CuspExtrapolation *>(c->ext)) {
        d.left_kind = 1;
        d.l0 = q->a0;
        d.l1 = q->b0;
        d.l2 = q->x0;
        d.right_kind = 0;
      } else if (auto *w = dynamic_cast<PowerExtrapolation *>(c->ext)) {
        d.left_kind = 0;
        d.right_kind = 2;
        d.r0 = w->amp;
        d.r1 = w->power;
      }
    }
    CubicSpline *c0 = splines[0];
    cudaStream_t s = host_api_stream();
    DevBuf<double> dp, dy, ddt, dout;
    DevBuf<SplineDesc> dsd;
    NAPMO_TRY_CUDA(dp.upload(points, 3 * npoint, s), "decomposition");
    NAPMO_TRY_CUDA(dy.upload(y, s), "decomposition");
    NAPMO_TRY_CUDA(ddt.upload(dt, s), "decomposition");
    NAPMO_TRY_CUDA(dsd.upload(sd, s), "decomposition");
    NAPMO_TRY_CUDA(dout.upload(output, npoint, s), "decomposition");
    decomposition_generic_kernel<<<(int)((npoint + 127) / 128), 128, 0, s>>>(
        (int)npoint, dp.p, center[0], center[1], center[2], dsd.p, (int)nspline, (int)lmax,
        c0->rtf->params(), c0->first_x, c0->last_x, c0->ext->has_tail() ? 1 : 0, dy.p,
        ddt.p, dout.p);
    NAPMO_TRY_CUDA(cudaGetLastError(), "decomposition");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(output, dout.p, npoint * sizeof(double),
                                   cudaMemcpyDeviceToHost, s),
                   "decomposition");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "decomposition");
    return kOk;
  });
}

void dot_multi_moments(long npoint, long nvector, double *data, double *points,
                       double *center, long lmax, long mtype, long *segments,
                       double *output, long nmoment) {
  guarded([&] {
    if (lmax < 0) return set_error(kInvalidArgument, "lmax can not be negative.");
    if (mtype < 1 || mtype > 4) return set_error(kInvalidArgument, "mtype should be 1, 2, 3 or 4.");
    if (lmax > kMaxLmax) return set_error(kNotSupported, "lmax too large");
    // the per-point polynomial work array holds (kMaxLmax + 1)^2 values
    if (nmoment < 1 || nmoment > (kMaxLmax + 1) * (kMaxLmax + 1) - 3)
      return set_error(kNotSupported, "too many moments");
    {
      long need = 1;
      if (mtype == 1)
        for (long l = 1; l <= lmax; ++l) need += (l + 1) * (l + 2) / 2;
      else if (mtype == 3)
        need = lmax + 1;
      else
        need = (lmax + 1) * (lmax + 1);
      if (need > (kMaxLmax + 1) * (kMaxLmax + 1) - 3 || nmoment > need)
        return set_error(kInvalidArgument, "nmoment does not match lmax and mtype");
    }
    std::vector<long> begin(1, 0);
    long nseg = 0;
    while (begin.back() < npoint) {
      begin.push_back(begin.back() + segments[nseg]);
      nseg++;
    }
    cudaStream_t s = host_api_stream();
    DevBuf<double> dd, dp, dpoly, dout;
    DevBuf<long> db;
    NAPMO_TRY_CUDA(dd.upload(data, nvector * npoint, s), "moments");
    NAPMO_TRY_CUDA(dp.upload(points, 3 * npoint, s), "moments");
    NAPMO_TRY_CUDA(dpoly.alloc(npoint * nmoment), "moments");
    NAPMO_TRY_CUDA(db.upload(begin, s), "moments");
    NAPMO_TRY_CUDA(dout.upload(output, nseg * nmoment, s), "moments");
    moments_poly_kernel<<<(int)((npoint + 127) / 128), 128, 0, s>>>(
        npoint, nvector, dd.p, dp.p, center[0], center[1], center[2], lmax, mtype, nmoment,
        dpoly.p);
    moments_sum_kernel<<<(int)((nseg * nmoment + 127) / 128), 128, 0, s>>>(nseg, db.p, nmoment,
                                                                          dpoly.p, dout.p);
    NAPMO_TRY_CUDA(cudaGetLastError(), "moments");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(output, dout.p, nseg * nmoment * sizeof(double),
                                   cudaMemcpyDeviceToHost, s),
                   "moments");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "moments");
    return kOk;
  });
}

// ------------------------------------------------------ device Poisson API
// Coulomb potential of rho (device, grid->size) on the grid's own points:
// v (device) = sum_A sum_lm spline_lm(r_A) S_lm / r_A^l.  With `accumulate`
// nonzero v is added to.  Optional raw spline output for the Python API:
// raw_y / raw_dt (device) receive [atom][lsize][nrad] solution splines.
int napmo_gpu_poisson(BeckeGrid *g, const double *rho_dev, int lmax, double *v_dev,
                      int accumulate, double *raw_y, double *raw_dt, void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    PoissonPlan *p = nullptr;
    int st = grid_poisson_plan(g, lmax, s, &p);
    if (st) return st;
    st = run_poisson(g, p, rho_dev, v_dev, accumulate != 0, s, g->poisson_tol, nullptr, 0);
    if (st) return st;
    if (raw_y)
      NAPMO_TRY_CUDA(cudaMemcpyAsync(raw_y, p->raw_y.p, p->raw_y.n * sizeof(double),
                                     cudaMemcpyDeviceToDevice, s),
                     "poisson raw");
    if (raw_dt)
      NAPMO_TRY_CUDA(cudaMemcpyAsync(raw_dt, p->raw_dt.p, p->raw_dt.n * sizeof(double),
                                     cudaMemcpyDeviceToDevice, s),
                     "poisson raw");
    return kOk;
  });
}

// ------------------------------------------- numerical-orbital operators
// Kinetic operator of nAPMO's numerical orbitals (compute_kinetic,
// napmo/wavefunction/nkinetic.py:15-73): out[k] = scale * (-1/2 laplacian
// psi[k]) at the grid's points for nfunc functions (device, rows of ld >=
// size doubles), through the Lebedev projection of psi wb, the radial
// operator (1/r d2/dr2 r - l(l+1)/r^2) by finite differences
// (src/grid/radial.cpp:51-192) and the multipole evaluation.  Every atom must
// use the Chebyshev radial transform (nAPMO's default) with >= 8 points.
int napmo_gpu_kinetic(BeckeGrid *g, int lmax, int nfunc, const double *psi, long ld,
                      double scale, double *out, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(nfunc >= 0 && ld >= g->size, "nfunc < 0 or ld < grid size");
    if (nfunc == 0) return kOk;
    for (auto &L : g->layout)
      if (L.rt.kind != kRTChebyshev || L.nrad < 8)
        return set_error(kNotSupported,
                         "the kinetic operator needs Chebyshev radial grids of >= 8 points");
    cudaStream_t s = (cudaStream_t)stream;
    PoissonDev P;
    int st = operator_dev(g, lmax, s, &P);
    if (st) return st;
    for (int k = 0; k < nfunc; ++k) {
      NAPMO_TRY_CUDA(launch_poisson_project(P, psi + (long)k * ld, g->dev.wb, g->dev.w, s),
                     "project");
      NAPMO_TRY_CUDA(launch_kinetic_radial(P, -0.5 * scale, s), "kinetic radial");
      NAPMO_TRY_CUDA(launch_poisson_evaluate(P, g->size, g->dev.x, g->dev.y, g->dev.z,
                                             out + (long)k * ld, false, s),
                     "evaluate");
    }
    return kOk;
  });
}

// Becke-Dickson orbital corrections (compute_dpsi,
// napmo/wavefunction/ndpsi.py:15-89) of nfunc orbitals: for orbital k the
// source (phi doi - R) wb is projected per atom, every (l, m) solves
//   u'' + 2/r u' - 2/m_inv (l(l+1)/r^2 + <V_k wb>(r) - oi - doi) u
//       = -2/m_inv src_lm,   u = 0 at both ends,
// (<.> the spherical average over each radial shell) and out[k] is the sum
// of the solutions over atoms at every point.  phi, resid, vtot, out: device
// rows of ld doubles; doi, oi: host arrays of nfunc.  Uses the grid's Poisson
// tables and a workspace kept with them: calls on one grid must not overlap
// on the device.
int napmo_gpu_dpsi(BeckeGrid *g, int lmax, int nfunc, const double *phi, const double *resid,
                   const double *vtot, long ld, const double *doi, const double *oi,
                   double mass_inv, double *out, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(nfunc >= 0 && ld >= g->size, "nfunc < 0 or ld < grid size");
    NAPMO_REQUIRE(mass_inv != 0.0, "mass_inv must be nonzero");
    if (nfunc == 0) return kOk;
    cudaStream_t s = (cudaStream_t)stream;
    PoissonDev P;
    PoissonPlan *plan = nullptr;
    int st = operator_dev(g, lmax, s, &P, &plan);
    if (st) return st;
    long nshell = 0;
    for (auto &L : g->layout) nshell += L.nrad;
    const size_t rows = (size_t)P.nsys * P.lu_stride;
    const size_t bytes = (g->size + nshell + rows * (kW + kKL)) * sizeof(double) +
                         rows * sizeof(int);
    if (plan->bd_ws.n < bytes) {
      NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "Becke-Dickson workspace");
      NAPMO_TRY_CUDA(plan->bd_ws.alloc(bytes), "Becke-Dickson workspace");
    }
    double *src = (double *)plan->bd_ws.p;
    double *vsph = src + g->size;
    P.lu = vsph + nshell;
    P.lmul = P.lu + rows * kW;
    P.lpiv = (int *)(P.lmul + rows * kKL);
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < nfunc && e == cudaSuccess; ++k) {
      RadialOp op;
      op.fscale = -2.0 / mass_inv;
      op.ascale = -2.0 / mass_inv;
      op.vsph = vsph;
      op.e = oi[k];
      op.de = doi[k];
      op.zero_bc = true;
      e = launch_dpsi_source(g->size, phi + (long)k * ld, resid + (long)k * ld, doi[k], src, s);
      if (e == cudaSuccess) e = launch_poisson_project(P, src, g->dev.wb, g->dev.w, s);
      if (e == cudaSuccess)
        e = launch_shell_average(P, vtot + (long)k * ld, g->dev.wb, g->dev.w, vsph, s);
      if (e == cudaSuccess) e = launch_radial_factor(P, op, s);
      if (e == cudaSuccess) e = launch_radial_solve(P, op, s);
      if (e == cudaSuccess)
        e = launch_poisson_evaluate(P, g->size, g->dev.x, g->dev.y, g->dev.z,
                                    out + (long)k * ld, false, s);
    }
    NAPMO_TRY_CUDA(e, "Becke-Dickson correction");
    return kOk;
  });
}

// M[i][j] = sum_p A[i][p] B[j][p] wb[p] w[p] for i < n, j < m: nAPMO's
// get_operator_matrix (napmo/wavefunction/psi_numeric.py:406-424, each entry
// a BeckeGrid::integrate of psi_i O psi_j).  A, B device rows (lda, ldb), M
// device [n][m].
int napmo_gpu_operator_matrix(BeckeGrid *g, int n, int m, const double *A, long lda,
                              const double *B, long ldb, double *M, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(n >= 0 && m >= 0 && lda >= g->size && ldb >= g->size,
                  "negative size or leading dimension < grid size");
    if (n == 0 || m == 0) return kOk;
    NAPMO_TRY_CUDA(launch_operator_matrix(g->size, n, m, A, lda, B, ldb, g->dev.wb, g->dev.w,
                                          M, (cudaStream_t)stream),
                   "operator matrix");
    return kOk;
  });
}

// k Poisson solves on the grid: v[j] = V_H[rho[j]] for device rows of
// ld >= size doubles, with the grid's truncation tolerance.
int napmo_gpu_poisson_many(BeckeGrid *g, int k, const double *rho_dev, long ld, int lmax,
                           double *v_dev, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(k >= 0 && ld >= g->size, "k < 0 or ld < grid size");
    cudaStream_t s = (cudaStream_t)stream;
    PoissonPlan *p = nullptr;
    int st = grid_poisson_plan(g, lmax, s, &p);
    if (st) return st;
    return run_poisson_many(g, p, k, rho_dev, ld, v_dev, s, g->poisson_tol, nullptr, 0);
  });
}

// Truncation tolerance (a.u., >= 0) of the grid's Poisson potential
// evaluation.  0 (the default) evaluates every (l, m) up to lmax at every
// pair, as nAPMO's evaluation does (src/horton/evaluate.cpp:129-220).  tol > 0
// lets each (atom, radial interval) bucket drop its highest l-blocks when the
// sum of their bounds (Racah-normalised harmonics: |sum_m c_lm S_lm| <=
// ||c_l||) is at most tol, so every pair's potential changes by at most tol.
// Applies to later builds; a batch graph keeps the tolerance it was
// captured with.
int napmo_grid_set_poisson_tolerance(BeckeGrid *g, double tol) {
  return guarded([&] {
    NAPMO_REQUIRE(tol >= 0.0 && tol < 1.0, "Poisson tolerance must be in [0, 1)");
    g->poisson_tol = tol;
    return kOk;
  });
}

// Number of doubles of the raw spline output of napmo_gpu_poisson.
long napmo_poisson_raw_size(BeckeGrid *g, int lmax) {
  long total = 0;
  for (auto &L : g->layout) total += (long)(lmax + 1) * (lmax + 1) * L.nrad;
  return total;
}

// Becke weights for arbitrary points on the device (points SoA), grouped by
// owner atom through atom_offset (host, ncenter+1); origin/radii host arrays.
int napmo_gpu_becke_weights(int npoint, int ncenter, const double *x, const double *y,
                            const double *z, const double *origin, const double *radii,
                            const int *atom_offset, double *out, void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    BeckeGrid tmp;
    tmp.ncenter = ncenter;
    tmp.size = npoint;
    tmp.origin.assign(origin, origin + 3 * ncenter);
    tmp.radii.assign(radii, radii + ncenter);
    const int tri = ncenter * (ncenter + 1) / 2;
    std::vector<double> R(tri), A(tri);
    int off = 0;
    for (int i = 0; i < ncenter; ++i)
      for (int j = 0; j <= i; ++j) R[off++] = distance_ref(&origin[3 * i], &origin[3 * j]);
    off = 0;
    for (int i = 0; i < ncenter; ++i)
      for (int j = 0; j <= i; ++j) {
        double aux = (radii[i] - radii[j]) / (radii[i] + radii[j]);
        aux = aux / (aux * aux - 1.0);
        if (aux > 0.45) aux = 0.45;
        else if (aux < -0.45) aux = -0.45;
        A[off++] = aux;
      }
    DevBuf<double> dR, dA, dO;
    DevBuf<int> dOff;
    NAPMO_TRY_CUDA(dR.upload(R, s), "becke");
    NAPMO_TRY_CUDA(dA.upload(A, s), "becke");
    NAPMO_TRY_CUDA(dO.upload(origin, 3 * ncenter, s), "becke");
    NAPMO_TRY_CUDA(dOff.upload(atom_offset, ncenter + 1, s), "becke");
    cudaError_t e = launch_becke_weights(npoint, ncenter, x, y, z, dO.p, dR.p, dA.p, dOff.p,
                                         out, s);
    if (e == cudaErrorInvalidValue) return set_error(kNotSupported, "too many centres");
    NAPMO_TRY_CUDA(e, "becke");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "becke");
    return kOk;
  });
}

}  // extern "C"
