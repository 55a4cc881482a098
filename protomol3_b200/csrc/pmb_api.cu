// C ABI of libpmb200: systems (batches of periodic boxes), force terms and the device MD loop.
//
// Host-side set-up mirrors what the reference does once per force:
//   * alpha by bisection on erfc(alpha rc)/rc = accuracy
//     (mdl/interface/force/nonbonded/NonbondedPMEwaldSystemForce.h:520-537);
//   * self energy -alpha/sqrt(pi) sum q^2 and charged-system energy (:555-575);
//   * lattice vectors for boxes smaller than twice the cutoff
//     (topology/PeriodicBoundaryConditions.cpp:79-106);
//   * grid tables exp(-pi^2 m^2/alpha^2) and the B-spline moduli (Grid.h:498-600).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

// PME transform work items per CTA (z-lines <= 16; rows / columns capped by the line buffer).
#ifndef PME_ZLINES
#define PME_ZLINES 8
#endif
#ifndef PME_YROWS
#define PME_YROWS 4
#endif
#ifndef PME_XCOLS
#define PME_XCOLS 8
#endif

#include "../../include/pmb200.h"
#include "pmb_internal.h"

namespace pmb {
static thread_local std::string g_err;
void set_error(const std::string &m) { g_err = m; }
}  // namespace pmb

using namespace pmb;

namespace {

#define CK(expr)                                                                          \
  do {                                                                                    \
    cudaError_t _e = (expr);                                                              \
    if (_e != cudaSuccess) {                                                              \
      set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));                      \
      return PMB_ERR_CUDA;                                                                \
    }                                                                                     \
  } while (0)

int fail(int code, const std::string &m) {
  set_error(m);
  return code;
}

struct Allocs {
  std::vector<void *> ptrs;
  size_t bytes = 0;  // device bytes held
  ~Allocs() {
    for (void *p : ptrs) cudaFree(p);
  }
  template <typename T>
  T *get(size_t n, bool zero = true) {
    void *p = nullptr;
    if (n == 0) n = 1;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    if (zero) cudaMemset(p, 0, n * sizeof(T));
    ptrs.push_back(p);
    bytes += n * sizeof(T);
    return static_cast<T *>(p);
  }
};

template <typename T>
int upload(Allocs &a, T *&dst, const std::vector<T> &src) {
  dst = a.get<T>(src.size(), false);
  if (!dst) return fail(PMB_ERR_CUDA, "cudaMalloc failed");
  if (!src.empty()) CK(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return PMB_OK;
}

double poly5h(double ar) {
  double t = 1.0 / (1.0 + 0.3275911 * ar);
  return t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
}

void bspline_h(int P, double w, double *th) {
  if (P == 2) {
    th[1] = w;
    th[0] = 1.0 - w;
    return;
  }
  th[P - 1] = 0.0;
  th[1] = w;
  th[0] = 1.0 - w;
  for (int k = 2; k < P - 1; k++) {
    double div = 1.0 / k;
    th[k] = div * w * th[k - 1];
    for (int j = 1; j < k; j++) th[k - j] = div * ((w + j) * th[k - j - 1] + ((double)(k + 1 - j) - w) * th[k - j]);
    th[0] = div * (1 - w) * th[0];
  }
  double div = 1.0 / (P - 1.0);
  th[P - 1] = div * w * th[P - 2];
  for (int j = 1; j < P - 1; j++) th[P - 1 - j] = div * ((w + j) * th[P - j - 2] + ((double)(P - j) - w) * th[P - 1 - j]);
  th[0] = div * (1 - w) * th[0];
}

double alpha_bisect(double rc, double acc) {
  double a = 1.0;
  while (std::erfc(a * rc) / rc >= acc) a *= 2.0;
  double lo = 0.0, hi = a;
  for (int i = 0; i < 100; ++i) {
    a = 0.5 * (lo + hi);
    if (std::erfc(a * rc) / rc >= acc) lo = a;
    else hi = a;
  }
  return a;
}

// Lattice vectors with |v| <= 2 rc, (0,0,0) first, by increasing norm.
std::vector<double> lattice_vectors(const double L[3], double rc) {
  int bk = (int)std::floor(rc / L[0] + 1.0), bl = (int)std::floor(rc / L[1] + 1.0),
      bm = (int)std::floor(rc / L[2] + 1.0);
  std::vector<std::pair<double, std::vector<double>>> v;
  for (int k = -bk; k <= bk; k++)
    for (int l = -bl; l <= bl; l++)
      for (int m = -bm; m <= bm; m++)
        if (k || l || m) {
          std::vector<double> c = {L[0] * k, L[1] * l, L[2] * m};
          double n2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
          if (std::sqrt(n2) <= 2 * rc) v.push_back({n2, c});
        }
  std::stable_sort(v.begin(), v.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
  std::vector<double> out = {0, 0, 0};
  for (auto &e : v) out.insert(out.end(), e.second.begin(), e.second.end());
  return out;
}

bool factor235(int n, std::vector<int> &rad) {
  rad.clear();
  while (n % 4 == 0) { rad.push_back(4); n /= 4; }
  while (n % 2 == 0) { rad.push_back(2); n /= 2; }
  while (n % 3 == 0) { rad.push_back(3); n /= 3; }
  while (n % 5 == 0) { rad.push_back(5); n /= 5; }
  return n == 1;
}

SwitchDev make_switch(int kind, double switchon, double cutoff) {
  SwitchDev w;
  std::memset(&w, 0, sizeof(w));
  w.kind = kind;
  w.rc2 = cutoff * cutoff;
  w.ron2 = switchon * switchon;
  double d = cutoff * cutoff - switchon * switchon;
  if (kind == SW_C2) {
    w.s1 = 1.0 / (d * d * d);
    w.s2 = cutoff * cutoff - 3.0 * switchon * switchon;
    w.s3 = 4.0 / (d * d * d);
  }
  w.c15_1 = 1.5 / cutoff;
  w.c05_3 = 0.5 / (cutoff * cutoff * cutoff);
  w.c15_3 = 1.5 / (cutoff * cutoff * cutoff);
  return w;
}

void switch_host(const SwitchDev &w, double r2, double &val, double &der) {
  if (w.kind == SW_C2) {
    der = 0.0;
    if (r2 > w.rc2) val = 0.0;
    else if (r2 >= w.ron2) {
      double c2 = w.rc2 - r2, c4 = c2 * (w.s2 + 2.0 * r2);
      val = w.s1 * (c2 * c4);
      der = w.s3 * (c2 * c2 - c4);
    } else val = 1.0;
  } else if (w.kind == SW_C1) {
    if (r2 > w.rc2) { val = 0; der = 0; return; }
    double d = std::sqrt(r2);
    val = 1.0 - d * (w.c15_1 - r2 * w.c05_3);
    der = -w.c15_1 / d + d * w.c15_3;
  } else {
    der = 0.0;
    val = r2 > w.rc2 ? 0.0 : 1.0;
  }
}

int valid_switch(int k) { return k == SW_CUTOFF || k == SW_C1 || k == SW_C2; }

}  // namespace

// ================================================================================== system
// Threads that add the forces of a host-pointer evaluation into the caller's array while the
// device->host copies land piece by piece: worker k (the calling thread is worker 0) waits for
// each piece's event and adds its share of the piece.  Between evaluations the workers sleep on
// a condition variable (spinning would take cores from the caller's own threads).
struct AddPool {
  int nthreads = 1, device = 0;
  std::vector<std::thread> th;
  std::mutex mu;
  std::condition_variable cv;
  std::atomic<long long> gen{0};
  std::atomic<int> pending{0};
  std::atomic<bool> stop{false};
  // the job
  double *dst = nullptr;
  const double *src = nullptr;
  long long n = 0, chunk = 0;
  int nchunks = 0;
  const cudaEvent_t *ev = nullptr;  // ev[c]: piece c has landed

  void part(int k) {
    for (int c = 0; c < nchunks; c++) {
      cudaEventSynchronize(ev[c]);
      const long long b0 = c * chunk, b1 = std::min(n, b0 + chunk), len = b1 - b0;
      const long long q0 = b0 + len * k / nthreads, q1 = b0 + len * (k + 1) / nthreads;
      double *__restrict__ d = dst;
      const double *__restrict__ s = src;
      for (long long i = q0; i < q1; i++) d[i] += s[i];
    }
  }
  void worker(int k) {
    cudaSetDevice(device);
    long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop.load() || gen.load(std::memory_order_acquire) != seen; });
        if (stop) return;
        seen = gen.load(std::memory_order_acquire);
      }
      part(k);
      pending.fetch_sub(1, std::memory_order_acq_rel);
    }
  }
  void start(int threads, int dev) {
    nthreads = threads;
    device = dev;
    for (int k = 1; k < nthreads; k++) th.emplace_back([this, k] { worker(k); });
  }
  // dst[0..n) += src[0..n), piece c of `chunk` elements once ev[c] has completed
  void run(double *d, const double *s, long long n_, long long chunk_, int nchunks_, const cudaEvent_t *ev_) {
    dst = d;
    src = s;
    n = n_;
    chunk = chunk_;
    nchunks = nchunks_;
    ev = ev_;
    pending.store(nthreads - 1, std::memory_order_release);
    {
      std::lock_guard<std::mutex> lk(mu);
      gen.fetch_add(1, std::memory_order_acq_rel);
    }
    cv.notify_all();
    part(0);
    while (pending.load(std::memory_order_acquire) > 0) std::this_thread::yield();
  }
  ~AddPool() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv.notify_all();
    for (std::thread &t : th) t.join();
  }
};

// A host-pointer evaluation captured as a CUDA graph: the force passes, the conversions and the
// device->host copies with their events, for one force set and virial flag.
struct EvalGraph {
  std::vector<unsigned long long> ids;
  int virial = 0;
  bool direct = false;  // forces added on the device to the caller's uploaded array (no host add)
  // page-locked caller arrays whose copies are nodes of the graph (null: copies outside it)
  const double *hpos = nullptr;
  double *hf = nullptr;
  long long gen = -1;  // list storage generation it was captured with
  double rlist = 0.0;
  bool used_list = false;
  cudaGraphExec_t exec = nullptr;
};

struct pmb_system {
  int precision = 0, nbox = 0, natoms = 0, ntypes = 0;
  cudaStream_t stream = nullptr;
  // second stream (higher priority) for the forces that run beside the pair kernel, with the
  // events that fork it from and join it to the system stream
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_slots = nullptr, ev_join = nullptr;
  bool own_stream = false;
  Allocs a;
  std::vector<BoxDev> hbox;
  std::vector<int> h_atom_box;
  std::vector<double> h_charge, h_lj, h_mass;
  std::vector<int> h_excl_pairs, h_excl_kind;  // global indices
  double coulomb_scaling = 1.0;
  BoxDev *d_box = nullptr;
  int *d_atom_box = nullptr, *d_type = nullptr, *d_mol = nullptr;
  double *d_pos = nullptr, *d_charge = nullptr, *d_mass = nullptr, *d_lj = nullptr;
  bool have_pos = false;  // positions were uploaded at least once (evaluate, profile, set_state)
  int *d_excl_start = nullptr, *d_excl_partner = nullptr, *d_excl_kindc = nullptr;
  int *d_excl_pairs = nullptr, *d_excl_kind = nullptr;
  BondedDev bonded{};
  long long *d_facc = nullptr, *d_eacc = nullptr;
  double *d_fout = nullptr, *d_eout = nullptr;
  double *h_fout = nullptr, *h_eout = nullptr;  // pinned
  int *h_status = nullptr;                      // pinned
  // host-pointer evaluations: the device->host copies go in EVAL_CHUNKS pieces, each followed by
  // an event, so that the host adds one piece while the next is in flight
  static constexpr int EVAL_CHUNKS = 4;
  cudaEvent_t ev_out[EVAL_CHUNKS + 1] = {};
  double eval_ms[3] = {0.0, 0.0, 0.0};  // last pmb_evaluate: enqueue, wait, accumulate (host ms)
  bool last_used_list = false;          // the last evaluation ran the list kernels
  bool eval_graph = true;               // host-pointer evaluations replay captured graphs
  AddPool *add_pool = nullptr;          // made at the first large host-pointer evaluation
  // host-pointer evaluations whose force array is page-locked: the array goes up on its own copy
  // stream once the positions have landed (the copy overlaps the force kernels), the device adds
  // the new forces to it and the sum comes back straight into the caller's array
  double *d_fin = nullptr;
  cudaStream_t copy = nullptr;
  cudaEvent_t ev_pos = nullptr, ev_fin = nullptr;
  std::vector<EvalGraph> eval_graphs;   // at most EVAL_GRAPHS, most recent last
  static constexpr int EVAL_GRAPHS = 4;
  // neighbour list
  bool nb_ready = false;
  double nb_cutoff = 0.0;    // radius the list storage is sized for
  double nb_build_rl = -1.0; // radius the current list was built with
  double skin = 0.8;         // list radius = pair cutoff + skin
  bool vacuum = false;       // boxes stand in for vacuum: evaluations check the extent
  double sort_cell = 2.4;    // smallest edge of a sort cell (A)
  int pair_ctas = 0;         // resident CTAs per SM of the pair kernel (0: as many as fit)
  NbListDev nb{};
  Allocs nba;
  long long nb_gen = 0;      // list storage and pair launch generation: graphs captured before a
                             // reallocation (or a change of the pair kernel's CTAs per SM) hold
                             // the old buffers (or launch shape) and are captured again
  int n_bonded = 0;
  // stage profiler: events recorded between launches when non-null
  std::vector<std::pair<std::string, cudaEvent_t>> *prof = nullptr;
  void *flush_buf = nullptr;  // > L2 scratch for cold-cache profiling

  SystemDev dev() const {
    SystemDev s;
    s.nbox = nbox;
    s.natoms = natoms;
    s.box = d_box;
    s.atom_box = d_atom_box;
    s.pos = d_pos;
    s.charge = d_charge;
    s.type = d_type;
    s.molecule = d_mol;
    s.excl_start = d_excl_start;
    s.excl_partner = d_excl_partner;
    s.excl_kind = d_excl_kindc;
    s.facc = d_facc;
    s.eacc = d_eacc;
    return s;
  }
  ~pmb_system() {
    delete add_pool;
    if (copy) cudaStreamDestroy(copy);
    if (ev_pos) cudaEventDestroy(ev_pos);
    if (ev_fin) cudaEventDestroy(ev_fin);
    for (EvalGraph &g : eval_graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    for (cudaEvent_t e : ev_out)
      if (e) cudaEventDestroy(e);
    if (flush_buf) cudaFree(flush_buf);
    if (h_fout) cudaFreeHost(h_fout);
    if (h_eout) cudaFreeHost(h_eout);
    if (h_status) cudaFreeHost(h_status);
    if (own_stream && stream) cudaStreamDestroy(stream);
    if (side) cudaStreamDestroy(side);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_slots) cudaEventDestroy(ev_slots);
    if (ev_join) cudaEventDestroy(ev_join);
  }
};

struct pmb_force {
  unsigned long long id = 0;  // unique over the process (keys the captured evaluations)
  pmb_system *sys = nullptr;
  pmb_force_desc d{};
  int kind = 0;
  // PME
  double alpha = 0.0;
  Allocs a;
  PmeDev pm{};
  std::vector<PmeBoxPlan> plans;
  std::vector<double> const_e;  // [nbox * ACC_PER_BOX] self / charged / self-image energies
  std::vector<double> const_vir;
  double *d_lattice = nullptr;
};

namespace {

// Sort cells per axis of a box edge: the largest power of two (at most 512) whose cells are at
// least min_edge long.
int sort_cells(double edge, double min_edge) {
  int nc = 1;
  while (nc < 512 && edge / (2 * nc) >= min_edge) nc *= 2;
  return nc;
}

// Neighbour-list storage sized for list cutoff rl.
int nblist_alloc(pmb_system *s, double rl) {
  cudaStreamSynchronize(s->stream);  // no kernel of the system may still read the old storage
  if (s->side) cudaStreamSynchronize(s->side);
  s->nb_gen++;
  s->nba.~Allocs();
  new (&s->nba) Allocs();
  NbListDev &nb = s->nb;
  std::memset(&nb, 0, sizeof(nb));
  int nblk = 0;
  for (auto &b : s->hbox) nblk += b.nblk;
  nb.nblk_total = nblk;
  nb.nslot = nblk * BLOCK;
  if ((long long)nblk * BLOCK >= JSAME) return fail(PMB_ERR_CAPACITY, "too many atoms for one system");
  std::vector<int> blk_box(nblk), jcap_off(nblk + 1, 0);
  long long tiles = 0;
  for (int bi = 0; bi < s->nbox; bi++) {
    const BoxDev &b = s->hbox[bi];
    // the box average, but at least a condensed-phase density (0.11 atoms/A^3): the atoms may
    // form a cluster inside a mostly empty box
    double V = b.L[0] * b.L[1] * b.L[2], rho = std::max(b.natoms / V, 0.11);
    double est = 1.5 * rho * (4.0 / 3.0) * M_PI * std::pow(rl + 8.0, 3) / 2.0 + 256.0;
    int cap = (int)std::min<double>(((b.natoms + 31) / 32) * 32.0, ((long long)est + 31) / 32 * 32.0);
    if (cap < 32) cap = 32;
    for (int k = 0; k < b.nblk; k++) {
      blk_box[b.blk0 + k] = bi;
      jcap_off[b.blk0 + k + 1] = cap;
      tiles += 1 + cap / 32;
    }
  }
  for (int k = 0; k < nblk; k++) jcap_off[k + 1] += jcap_off[k];
  tiles += (long long)s->nbox * (TILE_CHUNK - 1);  // each box's tiles start at a multiple of TILE_CHUNK
  if (tiles > 0x7fffffffLL || jcap_off[nblk] < 0) return fail(PMB_ERR_CAPACITY, "neighbour list too large");
  nb.tile_cap = (int)tiles;
  int *d_blk_box, *d_jcap;
  if (upload(s->nba, d_blk_box, blk_box) || upload(s->nba, d_jcap, jcap_off)) return PMB_ERR_CUDA;
  nb.blk_box = d_blk_box;
  nb.jcap_off = d_jcap;
  nb.blk_lo = s->nba.get<uint4>(nblk);
  nb.blk_hi = s->nba.get<uint4>(nblk);
  nb.nsblk = (nblk + 31) / 32;
  nb.sblk_lo = s->nba.get<uint4>(nb.nsblk);
  nb.sblk_hi = s->nba.get<uint4>(nb.nsblk);
  nb.blk_c = s->nba.get<uint4>(nblk);
  nb.blk_h = s->nba.get<uint4>(nblk);
  nb.sblk_c = s->nba.get<uint4>(nb.nsblk);
  nb.sblk_h = s->nba.get<uint4>(nb.nsblk);
  nb.jcount = s->nba.get<int>(nblk + 1);
  nb.jlist = s->nba.get<int>((size_t)jcap_off[nblk], false);
  nb.tile_off = s->nba.get<int>(nblk + 1);
  nb.tile_start = s->nba.get<int>(nblk + 1);
  nb.tile_blk = s->nba.get<int>(nb.tile_cap);
  nb.tile_k = s->nba.get<int>(nb.tile_cap);
  nb.status = s->nba.get<int>(4);
  nb.slot_orig = s->nba.get<int>(nb.nslot, false);
  if (nb.slot_orig) cudaMemset(nb.slot_orig, 0xff, sizeof(int) * nb.nslot);  // -1 padding
  nb.slot_fx = s->nba.get<uint4>(nb.nslot);
  nb.want_fp64 = s->precision == PMB_FP64;
  nb.slot_pq = nb.want_fp64 ? s->nba.get<double4>(nb.nslot) : nullptr;
  nb.slot_meta = s->nba.get<int4>(nb.nslot);
  nb.fslot = s->nba.get<long long>(3 * (size_t)nb.nslot);
  // sort bins
  std::vector<int> bin_box;
  for (int bi = 0; bi < s->nbox; bi++) {
    int ncm = std::max(s->hbox[bi].nc[0], std::max(s->hbox[bi].nc[1], s->hbox[bi].nc[2]));
    long long nk = (long long)ncm * ncm * ncm;
    bin_box.insert(bin_box.end(), (size_t)nk, bi);
  }
  nb.nkeys = (int)bin_box.size();
  int *d_bin_box;
  if (upload(s->nba, d_bin_box, bin_box)) return PMB_ERR_CUDA;
  nb.bin_box = d_bin_box;
  nb.key = s->nba.get<int>(s->natoms);
  nb.rank = s->nba.get<int>(s->natoms);
  nb.bin_count = s->nba.get<int>(nb.nkeys + 1);
  nb.bin_start = s->nba.get<int>(nb.nkeys + 1);
  int maxn = std::max(nb.nkeys, nblk) + 1;
  nb.scan_tmp = s->nba.get<int>(maxn / 4096 + 2);
  nb.xref = s->nba.get<double>(3 * (size_t)s->natoms);
  nb.ctl = s->nba.get<unsigned>(12);
  nb.vext = s->nba.get<int>(6 * (size_t)s->nbox);
  if (nb.vext) {
    std::vector<int> ext(6 * (size_t)s->nbox);
    for (size_t k = 0; k < ext.size(); k++) ext[k] = (k % 6) < 3 ? 0x7fffffff : (int)0x80000000;
    CK(cudaMemcpy(nb.vext, ext.data(), sizeof(int) * ext.size(), cudaMemcpyHostToDevice));
  }
  nb.half_skin2 = (float)(0.25 * s->skin * s->skin);
  nb.nbox = s->nbox;
  nb.box_d2 = s->nba.get<unsigned>(s->nbox);
  nb.box_rb = s->nba.get<unsigned>(s->nbox);
  nb.box_shift = s->nba.get<int>(s->nbox);
  {
    std::vector<int> order(s->nbox);
    for (int b = 0; b < s->nbox; b++) order[b] = b;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return s->hbox[a].blk0 < s->hbox[b].blk0; });
    int *d_order;
    if (upload(s->nba, d_order, order)) return PMB_ERR_CUDA;
    nb.box_order = d_order;
  }
  if (!nb.xref || !nb.ctl || !nb.vext || !nb.box_d2 || !nb.box_rb || !nb.box_shift || !nb.tile_start)
    return fail(PMB_ERR_CUDA, "cudaMalloc failed for the neighbour list");
  // {max displacement, rebuild, finished blocks, forced rebuild, builds (64-bit), pair chunk
  // counter and finished warps of the two pair launches, vacuum extent check}; first use builds
  // the list
  const unsigned ctl0[12] = {0u, 0u, 0u, 1u, 0u, 0u, 0u, 0u, 0u, 0u, s->vacuum ? 1u : 0u, 0u};
  CK(cudaMemcpy(nb.ctl, ctl0, sizeof(ctl0), cudaMemcpyHostToDevice));
  s->nb_build_rl = -1.0;
  if (!nb.blk_lo || !nb.sblk_lo || !nb.sblk_hi || !nb.blk_c || !nb.blk_h || !nb.sblk_c || !nb.sblk_h || !nb.jlist || !nb.tile_blk || !nb.slot_meta || !nb.fslot ||
      !nb.scan_tmp || !nb.bin_start)
    return fail(PMB_ERR_CUDA, "cudaMalloc failed for the neighbour list");
  s->nb_cutoff = rl;
  s->nb_ready = true;
  // the zero fills above run on the legacy default stream; the system's streams are
  // non-blocking, so wait for that stream alone (other streams' work keeps running)
  CK(cudaStreamSynchronize(cudaStreamLegacy));
  return PMB_OK;
}

int ensure_nblist(pmb_system *s, double rl) {
  if (s->nb_ready && rl <= s->nb_cutoff) return PMB_OK;
  return nblist_alloc(s, rl);
}

double force_pair_cutoff(const pmb_force *f) {
  if (f->kind == PMB_FORCE_CUTOFF)
    return std::max(f->d.lj ? f->d.lj_cutoff : 0.0, f->d.coulomb ? f->d.coulomb_cutoff : 0.0);
  if (f->kind == PMB_FORCE_PME && f->d.real) return f->d.cutoff;
  return 0.0;
}

struct PairJob {
  PairParams p;
  const double *lattice;
};

PairParams base_params(const pmb_system *s, int virial) {
  PairParams p;
  std::memset(&p, 0, sizeof(p));
  p.ntypes = s->ntypes;
  p.coulomb_scaling = s->coulomb_scaling;
  p.virial = virial;
  return p;
}

// Pair jobs of a force set; a cutoff LJ-only force and a PME real-space term are fused into one
// launch (LJ + Ewald real space).
std::vector<PairJob> pair_jobs(pmb_system *s, pmb_force *const *fs, int n, int virial) {
  std::vector<PairJob> jobs;
  const pmb_force *ljonly = nullptr, *pme = nullptr;
  for (int i = 0; i < n; i++) {
    if (fs[i]->kind == PMB_FORCE_CUTOFF && fs[i]->d.lj && !fs[i]->d.coulomb && !ljonly) ljonly = fs[i];
    if (fs[i]->kind == PMB_FORCE_PME && fs[i]->d.real && !pme) pme = fs[i];
  }
  const bool fuse = ljonly && pme;
  for (int i = 0; i < n; i++) {
    const pmb_force *f = fs[i];
    if (f->kind == PMB_FORCE_CUTOFF) {
      if (fuse && f == ljonly) continue;
      PairJob j;
      j.p = base_params(s, virial);
      j.lattice = nullptr;
      j.p.do_lj = f->d.lj;
      j.p.coul_mode = f->d.coulomb ? 1 : 0;
      j.p.lj_sw = make_switch(f->d.lj_switch, f->d.lj_switchon, f->d.lj_cutoff);
      j.p.coul_sw = make_switch(f->d.coulomb_switch, f->d.coulomb_switchon, f->d.coulomb_cutoff);
      j.p.lj_cut2 = f->d.lj_cutoff * f->d.lj_cutoff;
      j.p.coul_cut2 = f->d.coulomb_cutoff * f->d.coulomb_cutoff;
      double rc = force_pair_cutoff(f);
      j.p.cut2 = rc * rc;
      jobs.push_back(j);
    } else if (f->kind == PMB_FORCE_PME && f->d.real) {
      PairJob j;
      j.p = base_params(s, virial);
      j.lattice = f->d_lattice;
      j.p.coul_mode = 2;
      j.p.coul_sw = make_switch(f->d.real_switch, 0.0, f->d.cutoff);
      j.p.coul_cut2 = f->d.cutoff * f->d.cutoff;
      j.p.alpha = f->alpha;
      j.p.a2pi = 2.0 * f->alpha / std::sqrt(M_PI);
      double rc = f->d.cutoff;
      if (fuse && f == pme) {
        j.p.do_lj = 1;
        j.p.lj_sw = make_switch(ljonly->d.lj_switch, ljonly->d.lj_switchon, ljonly->d.lj_cutoff);
        j.p.lj_cut2 = ljonly->d.lj_cutoff * ljonly->d.lj_cutoff;
        rc = std::max(rc, ljonly->d.lj_cutoff);
      }
      j.p.cut2 = rc * rc;
      jobs.push_back(j);
    }
  }
  return jobs;
}

void mark(void *ctx, const char *name) {
  pmb_system *s = static_cast<pmb_system *>(ctx);
  if (!s->prof) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, s->stream);
  s->prof->push_back({name, e});
}

// Enqueues every force of the set on the system stream; accumulators must be zero.
// The second (higher-priority) stream of the system and its fork / join events.
int ensure_side_stream(pmb_system *s) {
  if (s->side) return PMB_OK;
  int lo = 0, hi = 0;
  CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  CK(cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, hi));
  CK(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&s->ev_slots, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
  return PMB_OK;
}

// The neighbour-list radius a force set needs (pair cutoff + skin + a margin for the fixed-point
// culling), or 0 when no force of the set uses the list (no pair term, no PME reciprocal term).
double list_radius(pmb_system *s, pmb_force *const *fs, int n) {
  double rl = 0.0;
  bool need = false;
  for (int i = 0; i < n; i++) {
    rl = std::max(rl, force_pair_cutoff(fs[i]));
    need |= pair_jobs(s, fs + i, 1, 0).size() > 0 || (fs[i]->kind == PMB_FORCE_PME && fs[i]->d.reciprocal);
  }
  return need ? std::max(rl, 1.0) + s->skin + 1e-3 : 0.0;
}

int enqueue_forces(pmb_system *s, pmb_force *const *fs, int n, int virial) {
  SystemDev sd = s->dev();
  cudaStream_t st = s->stream;
  std::vector<PairJob> jobs = pair_jobs(s, fs, n, virial);
  bool need_pme_slots = false;
  for (int i = 0; i < n; i++) need_pme_slots |= fs[i]->kind == PMB_FORCE_PME && fs[i]->d.reciprocal;
  const bool need_list = !jobs.empty() || need_pme_slots;
  s->last_used_list = need_list;
  // PME, exclusion corrections and bonded terms run on the side stream beside the list build and
  // the pair kernel (every sum is an integer atomic, so the interleaving does not change a bit):
  // the corrections and bonded terms from the start, the PME chain once this step's slot records
  // are packed.  The stage profiler keeps everything in one stream to time each stage.
  bool others = false;
  for (int i = 0; i < n; i++) others |= fs[i]->kind == PMB_FORCE_PME || fs[i]->kind == PMB_FORCE_BONDED;
  bool split = !s->prof && !jobs.empty() && others && st != cudaStreamLegacy;
  if (split && !s->side) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) split = false;  // created outside a capture only
    else if (int rc = ensure_side_stream(s)) return rc;
  }
  cudaStream_t so = st;
  if (split) {
    CK(cudaEventRecord(s->ev_fork, st));
    CK(cudaStreamWaitEvent(s->side, s->ev_fork, 0));
    so = s->side;
  }
  auto launch_recip = [&](pmb_force *f) {
    f->pm.virial = virial;
    pme_recip_launch(sd, s->nb, f->pm, so, mark, s);
  };
  auto launch_atom_terms = [&](pmb_force *f) {  // exclusion corrections, bonded: no list needed
    if (f->kind == PMB_FORCE_PME && f->d.correction) {
      f->pm.virial = virial;
      pme_correction_launch(sd, f->pm, s->d_excl_pairs, s->d_excl_kind, (int)s->h_excl_kind.size(),
                            s->coulomb_scaling, so);
      mark(s, "pme_correction");
    } else if (f->kind == PMB_FORCE_BONDED) {
      BondedDev b = s->bonded;
      b.virial = virial;
      bonded_launch(sd, b, so);
      mark(s, "bonded");
    }
  };
  if (split)
    for (int i = 0; i < n; i++) launch_atom_terms(fs[i]);
  if (need_list) {
    const double rlist = list_radius(s, fs, n);
    int rc = ensure_nblist(s, rlist);
    if (rc) return rc;
    if (rlist != s->nb_build_rl) {  // a list built for another radius cannot be reused
      CK(cudaMemsetAsync(s->nb.ctl + 3, 1, 1, st));
      s->nb_build_rl = rlist;
    }
    nblist_sort(sd, s->nb, st);
    if (split && need_pme_slots) {
      CK(cudaEventRecord(s->ev_slots, st));
      CK(cudaStreamWaitEvent(s->side, s->ev_slots, 0));
      for (int i = 0; i < n; i++)
        if (fs[i]->kind == PMB_FORCE_PME && fs[i]->d.reciprocal) launch_recip(fs[i]);
    }
    nblist_lists(sd, s->nb, rlist, st);
    mark(s, "nblist");
  }
  if (!split)
    for (int i = 0; i < n; i++) {
      if (fs[i]->kind == PMB_FORCE_PME && fs[i]->d.reciprocal) launch_recip(fs[i]);
      launch_atom_terms(fs[i]);
    }
  for (size_t q = 0; q < jobs.size(); q++) {
    const PairJob &j = jobs[q];
    PairLaunch pl;
    pl.precision = s->precision;
    pl.p = j.p;
    pl.lj = s->d_lj;
    pl.lattice = j.lattice;
    pl.multi = 0;
    pl.ctas_per_sm = s->pair_ctas;
    pl.blk_lo = 0;
    pl.blk_hi = s->nb.nblk_total;
    pl.wslot = 0;
    int split_blk = -1;  // first block of the lattice-image suffix
    if (j.p.coul_mode == 2 && j.lattice) {
      int first = s->nb.nblk_total, nmulti = 0;
      for (const BoxDev &b : s->hbox)
        if (b.multi_image) {
          pl.multi = 1;
          first = std::min(first, b.blk0);
          nmulti += b.nblk;
        }
      if (pl.multi && first > 0 && first + nmulti == s->nb.nblk_total) split_blk = first;
    }
    if (split_blk > 0) {
      // the boxes that need no lattice image on the faster instance, the rest (a suffix of the
      // tile map) on the lattice-image one, each with its own chunk counter
      PairLaunch pa = pl, pb = pl;
      pa.multi = 0;
      pa.blk_hi = split_blk;
      pb.blk_lo = split_blk;
      pb.wslot = 1;
      if (pair_launch(sd, s->nb, pa, st) || pair_launch(sd, s->nb, pb, st))
        return fail(PMB_ERR_UNSUPPORTED, "too many LJ types");
    } else if (pair_launch(sd, s->nb, pl, st)) {
      return fail(PMB_ERR_UNSUPPORTED, "too many LJ types");
    }
    mark(s, "pair");
  }
  if (split) {
    CK(cudaEventRecord(s->ev_join, so));
    CK(cudaStreamWaitEvent(st, s->ev_join, 0));
  }
  // slot-ordered pair forces -> facc (a plain read-modify-write: after the join)
  if (!jobs.empty()) pair_fold(sd, s->nb, st);
  CK(cudaGetLastError());
  return PMB_OK;
}

void add_const(pmb_force *const *fs, int n, int nbox, int virial, double *e) {
  for (int i = 0; i < n; i++) {
    if (fs[i]->kind != PMB_FORCE_PME || !fs[i]->d.correction) continue;
    for (int b = 0; b < nbox; b++) {
      e[b * ACC_PER_BOX + E_COUL] += fs[i]->const_e[b];
      if (virial)
        for (int k = 0; k < 9; k++) e[b * ACC_PER_BOX + E_VIR + k] += fs[i]->const_vir[b * 9 + k];
    }
  }
}

// Device->host copies of a host-pointer evaluation on the system stream (inside or outside a
// capture): status and energies, then the forces in EVAL_CHUNKS pieces, each followed by its
// event (external events, so that the host can wait on them when they come from a graph).
int enqueue_eval_copies(pmb_system *s, bool with_forces = true) {
  cudaStream_t st = s->stream;
  const long long nf = 3LL * s->natoms;
  const long long chunk = (nf + pmb_system::EVAL_CHUNKS - 1) / pmb_system::EVAL_CHUNKS;
  if (s->nb_ready) CK(cudaMemcpyAsync(s->h_status, s->nb.status, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(s->h_eout, s->d_eout, sizeof(double) * s->nbox * ACC_PER_BOX, cudaMemcpyDeviceToHost, st));
  CK(cudaEventRecordWithFlags(s->ev_out[0], st, cudaEventRecordExternal));
  for (int c = 0; c < pmb_system::EVAL_CHUNKS && with_forces; c++) {
    const long long b0 = c * chunk, b1 = std::min(nf, b0 + chunk);
    if (b1 > b0)
      CK(cudaMemcpyAsync(s->h_fout + b0, s->d_fout + b0, sizeof(double) * (b1 - b0), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecordWithFlags(s->ev_out[c + 1], st, cudaEventRecordExternal));
  }
  return PMB_OK;
}

// One host-pointer evaluation's device work (the positions are already on the device): from a
// CUDA graph of the force set, captured at its first use.  A graph is kept while the list
// storage it captured stays (generation) and the list radius is unchanged; the list storage and
// radius are settled before any capture, so a captured step neither allocates nor forces a
// rebuild on every replay.
int eval_graph_launch(pmb_system *s, pmb_force *const *fs, int n, int virial, bool direct,
                      const double *hpos = nullptr, double *hf = nullptr) {
  cudaStream_t st = s->stream;
  const double rlist = list_radius(s, fs, n);
  if (rlist > 0.0) {
    int rc = ensure_nblist(s, rlist);
    if (rc) return rc;
    if (rlist != s->nb_build_rl) {
      CK(cudaMemsetAsync(s->nb.ctl + 3, 1, 1, st));
      s->nb_build_rl = rlist;
    }
  }
  if (int rc = ensure_side_stream(s)) return rc;
  std::vector<unsigned long long> ids(n);
  for (int i = 0; i < n; i++) ids[i] = fs[i]->id;
  EvalGraph *g = nullptr;
  for (size_t k = 0; k < s->eval_graphs.size(); k++) {
    EvalGraph &e = s->eval_graphs[k];
    if (e.ids == ids && e.virial == virial && e.direct == direct && e.hpos == hpos && e.hf == hf &&
        e.gen == s->nb_gen && e.rlist == rlist) {
      std::rotate(s->eval_graphs.begin() + k, s->eval_graphs.begin() + k + 1, s->eval_graphs.end());
      g = &s->eval_graphs.back();
      break;
    }
  }
  if (!g) {
    cudaGraph_t graph = nullptr;
    const long long nf = 3LL * s->natoms;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    // the captured work; a failing call returns from here, and the capture is ended below either way
    auto body = [&]() -> int {
      if (hpos) CK(cudaMemcpyAsync(s->d_pos, hpos, sizeof(double) * nf, cudaMemcpyHostToDevice, st));
      if (hf) {
        // the caller's forces go up after the positions (the two uploads would share the link),
        // beside the force kernels
        CK(cudaEventRecord(s->ev_pos, st));
        CK(cudaStreamWaitEvent(s->copy, s->ev_pos, 0));
        CK(cudaMemcpyAsync(s->d_fin, hf, sizeof(double) * nf, cudaMemcpyHostToDevice, s->copy));
        CK(cudaEventRecord(s->ev_fin, s->copy));
      }
      SystemDev sd = s->dev();
      zero_accumulators(sd, st);
      int rc = enqueue_forces(s, fs, n, virial);
      if (rc) return rc;
      if (direct) {  // the caller's forces, uploaded beside the force kernels, are the base
        CK(cudaStreamWaitEvent(st, s->ev_fin, hf ? 0 : cudaEventWaitExternal));
        forces_to_double(sd, s->d_fout, st, s->d_fin);
      } else {
        forces_to_double(sd, s->d_fout, st);
      }
      energies_to_double(sd, nullptr, s->d_eout, st);
      rc = enqueue_eval_copies(s, !direct);
      if (rc) return rc;
      if (hf) {
        CK(cudaMemcpyAsync(hf, s->d_fout, sizeof(double) * nf, cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecordWithFlags(s->ev_out[1], st, cudaEventRecordExternal));
      }
      return PMB_OK;
    };
    const int rc = body();
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return rc ? rc : fail(PMB_ERR_CUDA, std::string("evaluation capture: ") + cudaGetErrorString(e));
    }
    EvalGraph ng;
    ng.ids = ids;
    ng.virial = virial;
    ng.direct = direct;
    ng.hpos = hpos;
    ng.hf = hf;
    ng.gen = s->nb_gen;
    ng.rlist = rlist;
    ng.used_list = s->last_used_list;
    e = cudaGraphInstantiate(&ng.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(PMB_ERR_CUDA, std::string("evaluation graph: ") + cudaGetErrorString(e));
    if ((int)s->eval_graphs.size() >= pmb_system::EVAL_GRAPHS) {
      cudaGraphExecDestroy(s->eval_graphs.front().exec);
      s->eval_graphs.erase(s->eval_graphs.begin());
    }
    s->eval_graphs.push_back(ng);
    g = &s->eval_graphs.back();
  }
  s->last_used_list = g->used_list;
  CK(cudaGraphLaunch(g->exec, st));
  return PMB_OK;
}

// True when both ends of the n doubles at p are page-locked host memory (cudaMallocHost,
// cudaHostAlloc or cudaHostRegister), which the copy engines read and write directly.
bool host_pinned(const double *p, long long n) {
  for (const double *q : {p, p + n - 1}) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (at.type != cudaMemoryTypeHost) return false;
  }
  return true;
}

// The status words as they were copied to s->h_status: capacity before non-finite positions
// (a retry with larger lists comes first).  Clears the device words that were set.
int status_code(pmb_system *s) {
  if (s->h_status[0] || s->h_status[1] || s->h_status[2] || s->h_status[3]) {
    cudaMemsetAsync(s->nb.status, 0, 4 * sizeof(int), s->stream);
    if (s->h_status[0] || s->h_status[1])
      return fail(PMB_ERR_CAPACITY, "neighbour list capacity exceeded (atoms denser than expected)");
    if (s->h_status[2]) return fail(PMB_ERR_NUMERIC, "non-finite position");
    return fail(PMB_ERR_STATE, "vacuum: the atoms spread over half a box edge; make the system again with "
                               "edges from pmb_vacuum_box");
  }
  return PMB_OK;
}

int check_status(pmb_system *s) {
  if (!s->nb_ready) return PMB_OK;
  CK(cudaMemcpyAsync(s->h_status, s->nb.status, 4 * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return status_code(s);
}

int grow_and_retry_needed(pmb_system *s) {
  // doubles the per-block list capacity by pretending a larger list cutoff
  return nblist_alloc(s, s->nb_cutoff * 1.26 + 1.0);
}

}  // namespace

// ======================================================================================= ABI
extern "C" {

const char *pmb_last_error(void) { return g_err.c_str(); }

int pmb_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

pmb_system *pmb_system_create(const pmb_box_desc *boxes, int n_boxes, int precision) {
  if (!boxes || n_boxes <= 0) return fail(PMB_ERR_ARG, "no boxes"), nullptr;
  if (precision != PMB_FP64 && precision != PMB_MIXED) return fail(PMB_ERR_ARG, "precision"), nullptr;
  if (pmb_device_count() <= 0) return fail(PMB_ERR_CUDA, "no CUDA device"), nullptr;
  pmb_system *s = new pmb_system();
  s->precision = precision;
  s->nbox = n_boxes;
  s->ntypes = boxes[0].n_types;
  if (s->ntypes <= 0 || s->ntypes > MAX_LJ_TYPES || !boxes[0].lj) {
    delete s;
    return fail(PMB_ERR_UNSUPPORTED, "1 <= n_types <= 32 required"), nullptr;
  }
  s->h_lj.assign(boxes[0].lj, boxes[0].lj + 4 * s->ntypes * s->ntypes);
  s->coulomb_scaling = boxes[0].coulomb_scaling;
  std::vector<int> type, mol, estart, epart, ekind, bonds, angles;
  std::vector<double> bk, br, ak, at, uk, ur;
  int blk = 0, key0 = 0, mol0 = 0;
  for (int bi = 0; bi < n_boxes; bi++) {
    const pmb_box_desc &d = boxes[bi];
    if (d.n_atoms <= 0 || !d.charge || !d.type || !d.molecule) {
      delete s;
      return fail(PMB_ERR_ARG, "box " + std::to_string(bi) + ": atoms, charge, type, molecule required"), nullptr;
    }
    if (d.n_types != s->ntypes ||
        std::memcmp(d.lj, s->h_lj.data(), sizeof(double) * s->h_lj.size()) != 0 ||
        d.coulomb_scaling != s->coulomb_scaling) {
      delete s;
      return fail(PMB_ERR_UNSUPPORTED, "all boxes of a system must share the LJ table and coulombScalingFactor"), nullptr;
    }
    BoxDev b;
    std::memset(&b, 0, sizeof(b));
    for (int k = 0; k < 3; k++) {
      if (!(d.box[k] > 0.0)) {
        delete s;
        return fail(PMB_ERR_ARG, "box edges must be positive"), nullptr;
      }
      b.L[k] = d.box[k];
      b.Lr[k] = 1.0 / d.box[k];
      double lo = -d.box[k] * 0.5, hi = d.box[k] * 0.5;
      b.H[k] = hi - lo;
      b.H2[k] = b.H[k] * 0.5;
      b.nc[k] = sort_cells(d.box[k], s->sort_cell);
    }
    b.D = std::min((d.box[0] * 0.5) * (d.box[0] * 0.5),
                   std::min((d.box[1] * 0.5) * (d.box[1] * 0.5), (d.box[2] * 0.5) * (d.box[2] * 0.5)));
    int ncm = std::max(b.nc[0], std::max(b.nc[1], b.nc[2]));
    b.nc[0] = b.nc[1] = b.nc[2] = ncm;  // one Morton space per box
    b.atom0 = s->natoms;
    b.natoms = d.n_atoms;
    b.blk0 = blk;
    b.nblk = (d.n_atoms + BLOCK - 1) / BLOCK;
    b.key0 = key0;
    b.nlat = 1;
    blk += b.nblk;
    key0 += ncm * ncm * ncm;
    s->hbox.push_back(b);
    int mmax = 0;
    for (int i = 0; i < d.n_atoms; i++) {
      if (d.type[i] < 0 || d.type[i] >= s->ntypes) {
        delete s;
        return fail(PMB_ERR_ARG, "atom type out of range"), nullptr;
      }
      s->h_atom_box.push_back(bi);
      s->h_charge.push_back(d.charge[i]);
      s->h_mass.push_back(d.mass ? d.mass[i] : 1.0);
      type.push_back(d.type[i]);
      mol.push_back(mol0 + d.molecule[i]);
      mmax = std::max(mmax, d.molecule[i] + 1);
    }
    mol0 += mmax;
    for (int k = 0; k < d.n_excl; k++) {
      int a1 = d.excl_pairs[2 * k], a2 = d.excl_pairs[2 * k + 1];
      if (a1 < 0 || a2 < 0 || a1 >= d.n_atoms || a2 >= d.n_atoms || a1 == a2) {
        delete s;
        return fail(PMB_ERR_ARG, "exclusion pair out of range"), nullptr;
      }
      s->h_excl_pairs.push_back(s->natoms + std::min(a1, a2));
      s->h_excl_pairs.push_back(s->natoms + std::max(a1, a2));
      s->h_excl_kind.push_back(d.excl_kind ? d.excl_kind[k] : 2);
    }
    for (int k = 0; k < d.n_bonds; k++)
      if (d.bonds[2 * k] < 0 || d.bonds[2 * k] >= d.n_atoms || d.bonds[2 * k + 1] < 0 ||
          d.bonds[2 * k + 1] >= d.n_atoms || d.bonds[2 * k] == d.bonds[2 * k + 1]) {
        delete s;
        return fail(PMB_ERR_ARG, "bond atom index out of range"), nullptr;
      }
    for (int k = 0; k < d.n_angles; k++)
      for (int c = 0; c < 3; c++)
        if (d.angles[3 * k + c] < 0 || d.angles[3 * k + c] >= d.n_atoms) {
          delete s;
          return fail(PMB_ERR_ARG, "angle atom index out of range"), nullptr;
        }
    for (int k = 0; k < d.n_bonds; k++) {
      bonds.push_back(s->natoms + d.bonds[2 * k]);
      bonds.push_back(s->natoms + d.bonds[2 * k + 1]);
      bk.push_back(d.bond_k[k]);
      br.push_back(d.bond_r0[k]);
    }
    for (int k = 0; k < d.n_angles; k++) {
      for (int c = 0; c < 3; c++) angles.push_back(s->natoms + d.angles[3 * k + c]);
      ak.push_back(d.angle_k[k]);
      at.push_back(d.angle_theta0[k]);
      uk.push_back(d.ub_k ? d.ub_k[k] : 0.0);
      ur.push_back(d.ub_r0 ? d.ub_r0[k] : 0.0);
    }
    s->natoms += d.n_atoms;
  }
  // exclusion CSR per atom (both directions)
  int N = s->natoms;
  estart.assign(N + 1, 0);
  size_t ne = s->h_excl_kind.size();
  for (size_t k = 0; k < ne; k++) {
    estart[s->h_excl_pairs[2 * k] + 1]++;
    estart[s->h_excl_pairs[2 * k + 1] + 1]++;
  }
  for (int i = 0; i < N; i++) estart[i + 1] += estart[i];
  epart.assign(2 * ne + 1, -1);
  ekind.assign(2 * ne + 1, 0);
  std::vector<int> fill(N, 0);
  for (size_t k = 0; k < ne; k++) {
    int a = s->h_excl_pairs[2 * k], b = s->h_excl_pairs[2 * k + 1];
    epart[estart[a] + fill[a]] = b;
    ekind[estart[a] + fill[a]++] = s->h_excl_kind[k];
    epart[estart[b] + fill[b]] = a;
    ekind[estart[b] + fill[b]++] = s->h_excl_kind[k];
  }
  // Slot blocks of the boxes in order of decreasing smallest edge (stable): boxes small enough to
  // need Ewald lattice images come last in the tile map, so the pair kernel's lattice-image
  // instance runs over that suffix alone.  Atoms keep the caller's order.
  {
    std::vector<int> order(s->nbox);
    for (int bi = 0; bi < s->nbox; bi++) order[bi] = bi;
    auto min_edge = [&](int bi) { return std::min(s->hbox[bi].L[0], std::min(s->hbox[bi].L[1], s->hbox[bi].L[2])); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return min_edge(a) > min_edge(b); });
    int b0 = 0;
    for (int bi : order) {
      s->hbox[bi].blk0 = b0;
      b0 += s->hbox[bi].nblk;
    }
  }
  int rc = 0;
  rc |= upload(s->a, s->d_box, s->hbox);
  rc |= upload(s->a, s->d_atom_box, s->h_atom_box);
  rc |= upload(s->a, s->d_charge, s->h_charge);
  rc |= upload(s->a, s->d_mass, s->h_mass);
  rc |= upload(s->a, s->d_type, type);
  rc |= upload(s->a, s->d_mol, mol);
  rc |= upload(s->a, s->d_lj, s->h_lj);
  rc |= upload(s->a, s->d_excl_start, estart);
  rc |= upload(s->a, s->d_excl_partner, epart);
  rc |= upload(s->a, s->d_excl_kindc, ekind);
  rc |= upload(s->a, s->d_excl_pairs, s->h_excl_pairs);
  rc |= upload(s->a, s->d_excl_kind, s->h_excl_kind);
  int *d_bonds, *d_angles;
  double *d_bk, *d_br, *d_ak, *d_at, *d_uk, *d_ur;
  rc |= upload(s->a, d_bonds, bonds);
  rc |= upload(s->a, d_bk, bk);
  rc |= upload(s->a, d_br, br);
  rc |= upload(s->a, d_angles, angles);
  rc |= upload(s->a, d_ak, ak);
  rc |= upload(s->a, d_at, at);
  rc |= upload(s->a, d_uk, uk);
  rc |= upload(s->a, d_ur, ur);
  s->bonded.nbonds = (int)bk.size();
  s->bonded.nangles = (int)ak.size();
  s->bonded.bonds = d_bonds;
  s->bonded.bond_k = d_bk;
  s->bonded.bond_r0 = d_br;
  s->bonded.angles = d_angles;
  s->bonded.angle_k = d_ak;
  s->bonded.angle_theta0 = d_at;
  s->bonded.ub_k = d_uk;
  s->bonded.ub_r0 = d_ur;
  s->d_pos = s->a.get<double>(3 * (size_t)N);
  s->d_facc = s->a.get<long long>(3 * (size_t)N);
  s->d_eacc = s->a.get<long long>((size_t)n_boxes * ACC_PER_BOX);
  s->d_fout = s->a.get<double>(3 * (size_t)N);
  s->d_eout = s->a.get<double>((size_t)n_boxes * ACC_PER_BOX);
  if (rc || !s->d_pos || !s->d_facc || !s->d_eacc || !s->d_fout || !s->d_eout ||
      cudaMallocHost(&s->h_fout, sizeof(double) * 3 * (size_t)N) != cudaSuccess ||
      cudaMallocHost(&s->h_eout, sizeof(double) * n_boxes * ACC_PER_BOX) != cudaSuccess ||
      cudaMallocHost(&s->h_status, sizeof(int) * 4) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    return fail(PMB_ERR_CUDA, "device allocation failed"), nullptr;
  }
  s->own_stream = true;
  return s;
}

int pmb_system_destroy(pmb_system *s) {
  if (!s) return PMB_OK;
  cudaDeviceSynchronize();
  delete s;
  return PMB_OK;
}

int pmb_system_set_stream(pmb_system *s, void *stream) {
  if (!s) return fail(PMB_ERR_ARG, "null system");
  if (s->own_stream && s->stream) {
    cudaStreamSynchronize(s->stream);
    cudaStreamDestroy(s->stream);
  }
  s->own_stream = false;
  s->stream = (cudaStream_t)stream;
  return PMB_OK;
}

int pmb_system_n_atoms(const pmb_system *s) { return s ? s->natoms : 0; }
int pmb_system_n_boxes(const pmb_system *s) { return s ? s->nbox : 0; }

int pmb_system_set_skin(pmb_system *s, double skin) {
  if (!s || !(skin >= 0.0) || skin > 5.0) return fail(PMB_ERR_ARG, "skin must be in [0, 5] A");
  cudaStreamSynchronize(s->stream);
  s->skin = skin;
  s->nb_ready = false;  // storage is sized for cutoff + skin
  return PMB_OK;
}

int pmb_system_set_tuning(pmb_system *s, const pmb_tuning *t) {
  if (!s || !t) return fail(PMB_ERR_ARG, "null argument");
  if (!(t->skin >= 0.0) || t->skin > 5.0) return fail(PMB_ERR_ARG, "skin must be in [0, 5] A");
  if (!(t->sort_cell >= 0.5) || t->sort_cell > 50.0) return fail(PMB_ERR_ARG, "sort_cell must be in [0.5, 50] A");
  if (t->pair_ctas_per_sm < 0 || t->pair_ctas_per_sm > 32) return fail(PMB_ERR_ARG, "pair_ctas_per_sm in [0, 32]");
  CK(cudaStreamSynchronize(s->stream));
  if (t->pair_ctas_per_sm != s->pair_ctas) s->nb_gen++;  // captured steps hold the old launch shape
  s->pair_ctas = t->pair_ctas_per_sm;
  if (t->skin != s->skin || t->sort_cell != s->sort_cell) {
    s->skin = t->skin;
    s->sort_cell = t->sort_cell;
    // sort cells and their key ranges per box, then the lists are sized again at next use
    int key0 = 0;
    for (BoxDev &b : s->hbox) {
      int ncm = 1;
      for (int k = 0; k < 3; k++) ncm = std::max(ncm, sort_cells(b.L[k], s->sort_cell));
      b.nc[0] = b.nc[1] = b.nc[2] = ncm;
      b.key0 = key0;
      key0 += ncm * ncm * ncm;
    }
    CK(cudaMemcpy(s->d_box, s->hbox.data(), sizeof(BoxDev) * s->hbox.size(), cudaMemcpyHostToDevice));
    s->nb_ready = false;
  }
  return PMB_OK;
}

int pmb_system_get_tuning(const pmb_system *s, pmb_tuning *t) {
  if (!s || !t) return fail(PMB_ERR_ARG, "null argument");
  t->skin = s->skin;
  t->sort_cell = s->sort_cell;
  t->pair_ctas_per_sm = s->pair_ctas;
  return PMB_OK;
}

int pmb_system_check(pmb_system *s) {
  if (!s) return fail(PMB_ERR_ARG, "null system");
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  const int rc = check_status(s);
  if (rc == PMB_ERR_CAPACITY) {
    if (grow_and_retry_needed(s)) return PMB_ERR_CUDA;
    return fail(PMB_ERR_CAPACITY, "neighbour list capacity exceeded; the lists were enlarged, evaluate again");
  }
  return rc;
}

int pmb_system_list_builds(pmb_system *s, long long *n) {
  if (!s || !n) return fail(PMB_ERR_ARG, "null argument");
  *n = 0;
  if (!s->nb_ready) return PMB_OK;
  unsigned long long v = 0;
  CK(cudaMemcpyAsync(&v, s->nb.ctl + 4, sizeof(v), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *n = (long long)v;
  return PMB_OK;
}

int pmb_system_list_tiles(pmb_system *s, long long *tiles) {
  if (!s || !tiles) return fail(PMB_ERR_ARG, "null argument");
  *tiles = 0;
  if (!s->nb_ready) return PMB_OK;
  int v = 0;
  CK(cudaMemcpyAsync(&v, s->nb.tile_start + s->nb.nblk_total, sizeof(v), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *tiles = v;
  return PMB_OK;
}

int pmb_system_evaluate_times(const pmb_system *s, double ms[3]) {
  if (!s || !ms) return fail(PMB_ERR_ARG, "null argument");
  for (int k = 0; k < 3; k++) ms[k] = s->eval_ms[k];
  return PMB_OK;
}

pmb_force *pmb_force_create(pmb_system *s, const pmb_force_desc *d) {
  if (!s || !d) return fail(PMB_ERR_ARG, "null argument"), nullptr;
  pmb_force *f = new pmb_force();
  static std::atomic<unsigned long long> next_id{1};
  f->id = next_id++;
  f->sys = s;
  f->d = *d;
  f->kind = d->kind;
  auto bad = [&](int code, const std::string &m) {
    delete f;
    fail(code, m);
    return (pmb_force *)nullptr;
  };
  if (d->kind == PMB_FORCE_CUTOFF) {
    if (!d->lj && !d->coulomb) return bad(PMB_ERR_ARG, "cutoff force needs LennardJones and/or Coulomb");
    if ((d->lj && (!valid_switch(d->lj_switch) || !(d->lj_cutoff > 0))) ||
        (d->coulomb && (!valid_switch(d->coulomb_switch) || !(d->coulomb_cutoff > 0))))
      return bad(PMB_ERR_ARG, "invalid switching function or cutoff");
    if ((d->lj && d->lj_switch == SW_C2 && !(d->lj_switchon >= 0 && d->lj_switchon < d->lj_cutoff)) ||
        (d->coulomb && d->coulomb_switch == SW_C2 &&
         !(d->coulomb_switchon >= 0 && d->coulomb_switchon < d->coulomb_cutoff)))
      return bad(PMB_ERR_ARG, "C2 switching function: 0 <= switchon < cutoff");
    return f;
  }
  if (d->kind == PMB_FORCE_BONDED) return f;
  if (d->kind != PMB_FORCE_PME) return bad(PMB_ERR_ARG, "unknown force kind");
  // ---- PME: NonbondedPMEwaldSystemForce::doMake checks (:1033-1058)
  if (d->order < 2 || (d->order % 2) != 0 || d->order > 8) return bad(PMB_ERR_ARG, "order > 1, even and <= 8");
  if (!(d->cutoff > 0)) return bad(PMB_ERR_ARG, "PMEwald cutoff > 0");
  if (!(d->accuracy > 0)) return bad(PMB_ERR_ARG, "PMEwald accuracy > 0");
  if (d->real && d->real_switch != SW_CUTOFF && d->real_switch != SW_C1)
    return bad(PMB_ERR_ARG, "PME real-space switching function must be Cutoff or C1");
  f->alpha = d->alpha > 0.0 ? d->alpha : alpha_bisect(d->cutoff, d->accuracy);
  const int nbox = s->nbox, P = d->order;
  f->const_e.assign(nbox, 0.0);
  f->const_vir.assign(9 * (size_t)nbox, 0.0);
  // constants per box
  SwitchDev rsw = make_switch(d->real_switch, 0.0, d->cutoff);
  std::vector<double> lat_all;
  for (int bi = 0; bi < nbox; bi++) {
    BoxDev &b = s->hbox[bi];
    double q2 = 0.0, q1 = 0.0;
    for (int i = b.atom0; i < b.atom0 + b.natoms; i++) {
      q2 += s->h_charge[i] * s->h_charge[i];
      q1 += s->h_charge[i];
    }
    double V = b.L[0] * b.L[1] * b.L[2];
    double self = -q2 * f->alpha / std::sqrt(M_PI);
    double charged = std::fabs(q1 * 0.00268283) > 1.0e-5 ? -M_PI / (2.0 * V * f->alpha * f->alpha) * q1 * q1 : 0.0;
    f->const_e[bi] = self + charged;
    f->const_vir[9 * bi + 0] += charged;
    f->const_vir[9 * bi + 4] += charged;
    f->const_vir[9 * bi + 8] += charged;
    if (d->real) {
      std::vector<double> lat = lattice_vectors(b.L, d->cutoff);
      int nl = (int)lat.size() / 3;
      b.lat0 = (int)lat_all.size() / 3;
      b.nlat = nl;
      b.multi_image = nl > 1;
      lat_all.insert(lat_all.end(), lat.begin(), lat.end());
      // i == j lattice images (realTerm with i == j): energy only, forces cancel
      double a2pi = 2.0 * f->alpha / std::sqrt(M_PI);
      for (int k = 1; k < nl; k++) {
        double r2 = lat[3 * k] * lat[3 * k] + lat[3 * k + 1] * lat[3 * k + 1] + lat[3 * k + 2] * lat[3 * k + 2];
        if (r2 > d->cutoff * d->cutoff) continue;
        double r = std::sqrt(r2), rr = 1.0 / r, ar = f->alpha * r;
        double g = std::exp(-ar * ar), e0 = poly5h(ar) * g * rr, f0 = (e0 + a2pi * g) * rr * rr, val, der;
        switch_host(rsw, r2, val, der);
        f0 = f0 * val - e0 * der;
        e0 = e0 * val;
        f->const_e[bi] += q2 * e0;
        for (int p = 0; p < 3; p++)
          for (int q = 0; q < 3; q++) f->const_vir[9 * bi + 3 * p + q] += q2 * f0 * lat[3 * k + p] * lat[3 * k + q];
      }
    }
  }
  if (d->real) {
    if (upload(f->a, f->d_lattice, lat_all)) return bad(PMB_ERR_CUDA, "upload failed");
    // (no kernel of the system may still read the box records)
    if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
        cudaMemcpy(s->d_box, s->hbox.data(), sizeof(BoxDev) * nbox, cudaMemcpyHostToDevice) != cudaSuccess)
      return bad(PMB_ERR_CUDA, "upload failed");
    s->nb_ready = false;  // list culling depends on multi_image
  }
  if (d->reciprocal) {
    std::vector<double2> tw;
    std::vector<float2> twf;
    std::vector<double> infl;
    std::vector<int> radix;
    std::vector<int4> zwork;
    std::vector<int4> ywork, xwork;
    long long g0 = 0, c0 = 0;
    const int lcap = pme_line_capacity();
    int zbuf = 1, lbuf = 1;
    std::vector<double> theta;
    double th0[8];
    bspline_h(P, 0.0, th0);
    for (int bi = 0; bi < nbox; bi++) {
      const BoxDev &b = s->hbox[bi];
      PmeBoxPlan pl;
      std::memset(&pl, 0, sizeof(pl));
      for (int k = 0; k < 3; k++) {
        int n = d->box_grids ? d->box_grids[3 * bi + k] : d->grid[k];
        std::vector<int> rad;
        if (n < P || n > 256 || !factor235(n, rad))
          return bad(PMB_ERR_UNSUPPORTED, "PME grid sizes must be >= order, <= 256 and of the form 2^a 3^b 5^c");
        pl.n[k] = n;
        pl.hr[k] = n / b.L[k];
        pl.mr[k] = 1.0 / b.L[k];
        pl.tw0[k] = (int)tw.size();
        for (int j = 0; j < n; j++) {
          double ang = -2.0 * M_PI * j / n;
          tw.push_back(make_double2(std::cos(ang), std::sin(ang)));
          twf.push_back(make_float2((float)std::cos(ang), (float)std::sin(ang)));
        }
        pl.rad0[k] = (int)radix.size();
        pl.nrad[k] = (int)rad.size();
        radix.insert(radix.end(), rad.begin(), rad.end());
        // influence factor B(m) exp(-pi^2 m^2/alpha^2) (Grid.h:523-571, dftmod :588-600)
        pl.inf0[k] = (int)infl.size();
        double fac = M_PI * M_PI / (f->alpha * f->alpha);
        for (int i = 0; i < n; i++) {
          int i0 = i <= n / 2 ? i : i - n;
          double m = i0 * (1.0 / b.L[k]);
          double ex = std::exp(-fac * (m * m));
          double sc = 0.0, ss = 0.0;
          for (int j = 0; j < P; j++) {
            double x = M_PI * 2.0 * i * j / (double)n;
            sc += th0[j] * std::cos(x);
            ss += th0[j] * std::sin(x);
          }
          infl.push_back(ex / (sc * sc + ss * ss));
        }
      }
      pl.grid0 = g0;
      pl.cgrid0 = c0;
      pl.piVr = 1.0 / (M_PI * b.L[0] * b.L[1] * b.L[2]);
      pl.fac = M_PI * M_PI / (f->alpha * f->alpha);
      g0 += (long long)pl.n[0] * pl.n[1] * pl.n[2];
      c0 += (long long)(pl.n[2] / 2 + 1) * pl.n[0] * pl.n[1];
      // small work items (PME_ZLINES z-lines = PME_ZLINES / 2 packed complex lines, PME_YROWS
      // y-lines, PME_XCOLS x-lines per CTA): many CTAs in flight hide the latency of the
      // shared-memory stages
      for (int x = 0; x < pl.n[0]; x++)
        for (int y0 = 0; y0 < pl.n[1]; y0 += PME_ZLINES) {
          const int cnt = std::min(PME_ZLINES, pl.n[1] - y0);
          zwork.push_back(make_int4(bi, x, y0, cnt));
          zbuf = std::max(zbuf, (cnt + 1) / 2 * pl.n[2]);
        }
      const int rows = std::max(1, std::min(PME_YROWS, lcap / pl.n[1])),
                cols = std::max(1, std::min(PME_XCOLS, lcap / pl.n[0]));
      lbuf = std::max(lbuf, std::max(rows * pl.n[1], cols * pl.n[0]));
      for (int kz = 0; kz <= pl.n[2] / 2; kz++) {
        for (int x0 = 0; x0 < pl.n[0]; x0 += rows) ywork.push_back(make_int4(bi, kz, x0, std::min(rows, pl.n[0] - x0)));
        for (int y0 = 0; y0 < pl.n[1]; y0 += cols) xwork.push_back(make_int4(bi, kz, y0, std::min(cols, pl.n[1] - y0)));
      }
      // influence function per half-spectrum point [kz][x][y] (Grid.h:236-341): B(m)
      // exp(-pi^2 m^2/alpha^2) / (pi V m^2), 0 at m = 0
      {
        const int nx = pl.n[0], ny = pl.n[1], nh = pl.n[2] / 2 + 1;
        const double *bx = infl.data() + pl.inf0[0], *by = infl.data() + pl.inf0[1],
                     *bz = infl.data() + pl.inf0[2];
        for (int kz = 0; kz < nh; kz++)
          for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) {
              double th = 0.0;
              if (i || j || kz) {
                const int i0 = i <= nx / 2 ? i : i - nx, j0 = j <= ny / 2 ? j : j - ny;
                const double mi = i0 * pl.mr[0], mj = j0 * pl.mr[1], mk = kz * pl.mr[2];
                const double m2 = mi * mi + mj * mj + mk * mk;
                th = bx[i] * by[j] * bz[kz] * pl.piVr / m2;
              }
              theta.push_back(th);
            }
      }
      f->plans.push_back(pl);
    }
    PmeDev &pm = f->pm;
    pm.nbox = nbox;
    pm.order = P;
    pm.precision = s->precision;
    pm.alpha = f->alpha;
    pm.a2pi = 2.0 * f->alpha / std::sqrt(M_PI);
    PmeBoxPlan *dplan;
    double2 *dtw;
    float2 *dtwf;
    double *dinf;
    int *drad;
    int4 *dz, *dy, *dx;
    int rc = 0;
    rc |= upload(f->a, dplan, f->plans);
    rc |= upload(f->a, dtw, tw);
    rc |= upload(f->a, dtwf, twf);
    rc |= upload(f->a, dinf, infl);
    if (s->precision) {
      std::vector<float> thf(theta.begin(), theta.end());
      float *dth;
      rc |= upload(f->a, dth, thf);
      pm.theta = dth;
    } else {
      double *dth;
      rc |= upload(f->a, dth, theta);
      pm.theta = dth;
    }
    rc |= upload(f->a, drad, radix);
    rc |= upload(f->a, dz, zwork);
    rc |= upload(f->a, dy, ywork);
    rc |= upload(f->a, dx, xwork);
    pm.plan = dplan;
    pm.twiddle = dtw;
    pm.twiddlef = dtwf;
    pm.infl = dinf;
    pm.radix = drad;
    pm.zwork = dz;
    pm.nzwork = (int)zwork.size();
    pm.ywork = dy;
    pm.nywork = (int)ywork.size();
    pm.xwork = dx;
    pm.nxwork = (int)xwork.size();
    pm.zbuf = zbuf;
    pm.lbuf = lbuf;
    // the warp-shuffle transforms take lines of 32 R points (R <= 5), the same R in every box
    auto warp_r = [&](int d) {
      int r = 0;
      for (size_t bi = 0; bi < f->plans.size(); bi++) {
        const int n = f->plans[bi].n[d];
        if (n % 32 != 0 || n / 32 > 5 || (r && n / 32 != r)) return 0;
        r = n / 32;
      }
      return r;
    };
    // (one row per warp of a 4-warp block, one column per warp of an 8-warp block)
    pm.wy = PME_YROWS <= 4 ? warp_r(1) : 0;
    pm.wx = PME_XCOLS * 32 <= PME_WX_THREADS ? warp_r(0) : 0;
    pm.wz = PME_ZLINES <= 8 ? warp_r(2) : 0;  // (two lines per warp of a 4-warp block)
    pm.qgrid = f->a.get<long long>(g0);
    pm.rgrid = s->precision ? (void *)f->a.get<float>(g0) : (void *)f->a.get<double>(g0);
    pm.cgrid = s->precision ? (void *)f->a.get<float2>(c0) : (void *)f->a.get<double2>(c0);
    if (rc || !pm.qgrid || !pm.rgrid || !pm.cgrid) return bad(PMB_ERR_CUDA, "PME allocation failed");
  } else {
    f->pm.alpha = f->alpha;
    f->pm.a2pi = 2.0 * f->alpha / std::sqrt(M_PI);
    f->pm.precision = s->precision;
  }
  return f;
}

int pmb_force_destroy(pmb_force *f) {
  if (f) {
    cudaDeviceSynchronize();
    delete f;
  }
  return PMB_OK;
}

int pmb_force_alpha(const pmb_force *f, double *alpha) {
  if (!f || !alpha) return fail(PMB_ERR_ARG, "null argument");
  *alpha = f->alpha;
  return PMB_OK;
}

int pmb_evaluate_device(pmb_system *s, pmb_force *const *fs, int n, const double *d_pos,
                        double *d_forces, double *d_energies, int virial) {
  if (!s || (n > 0 && !fs)) return fail(PMB_ERR_ARG, "null argument");
  for (int i = 0; i < n; i++)
    if (!fs[i] || fs[i]->sys != s) return fail(PMB_ERR_ARG, "force belongs to another system");
  cudaStream_t st = s->stream;
  if (d_pos && d_pos != s->d_pos) {
    CK(cudaMemcpyAsync(s->d_pos, d_pos, sizeof(double) * 3 * s->natoms, cudaMemcpyDeviceToDevice, st));
    s->have_pos = true;
  }
  if (!s->have_pos) return fail(PMB_ERR_STATE, "no positions on the device yet: pass positions");
  SystemDev sd = s->dev();
  zero_accumulators(sd, st);
  int rc = enqueue_forces(s, fs, n, virial);
  if (rc) return rc;
  if (d_forces) forces_to_double(sd, d_forces, st);
  if (d_energies) energies_to_double(sd, nullptr, d_energies, st);
  CK(cudaGetLastError());
  return PMB_OK;
}

int pmb_ewald_reciprocal(pmb_system *s, const double *pos, double alpha, double accuracy, double *forces,
                         double *energies, int virial) {
  if (!s || !pos) return fail(PMB_ERR_ARG, "null argument");
  if (!(accuracy > 0 && accuracy < 1)) return fail(PMB_ERR_ARG, "accuracy must lie in (0, 1)");
  for (int i = 0; i < 3 * s->natoms; i++)
    if (!std::isfinite(pos[i])) return fail(PMB_ERR_NUMERIC, "non-finite position");
  cudaStream_t st = s->stream;
  CK(cudaMemcpyAsync(s->d_pos, pos, sizeof(double) * 3 * s->natoms, cudaMemcpyHostToDevice, st));
  s->have_pos = true;
  Allocs tmp;  // a check path: scratch per call
  double *d_f = tmp.get<double>(3 * (size_t)s->natoms);
  if (!d_f) return fail(PMB_ERR_CUDA, "cudaMalloc failed for the Ewald sum");
  std::vector<double> hf(3 * (size_t)s->natoms, 0.0);
  for (int bi = 0; bi < s->nbox; bi++) {
    const BoxDev &b = s->hbox[bi];
    // NonbondedFullEwaldSystemForce::initialize (NonbondedFullEwaldSystemForce.h:590-660), with the
    // box's volume and reciprocal edges as PeriodicBoundaryConditions::set forms them
    const double lx = b.L[0], ly = b.L[1], lz = b.L[2];
    const double V = (lx * ly) * lz, Vr = 1.0 / V;
    const double lxr = (ly * lz) / (lx * (ly * lz)), lyr = (lz * lx) / (ly * (lz * lx)),
                 lzr = (lx * ly) / (lz * (lx * ly));
    const double a = alpha > 0 ? alpha : std::sqrt(M_PI) * std::pow(5.5 * b.natoms / (V * V), 1.0 / 6.0);
    const double a2r = 1.0 / (a * a), fac = 1.0 / (4.0 * a * a);
    const double p = -std::log(accuracy);
    const double kc = 2.0 * a * std::sqrt(p), kc2 = kc * kc;
    const int hmax = (int)std::floor(kc / (2.0 * M_PI) * lx), kmax = (int)std::floor(kc / (2.0 * M_PI) * ly),
              lmax = (int)std::floor(kc / (2.0 * M_PI) * lz);
    std::vector<double3> kv;
    std::vector<double> ksq, bk, ak;
    for (int h = 0; h <= hmax; h++) {
      const double kx = 2.0 * M_PI * h * lxr;
      for (int k = (h == 0 ? 0 : -kmax); k <= kmax; k++) {
        const double ky = 2.0 * M_PI * k * lyr;
        for (int l = (h == 0 && k == 0 ? 1 : -lmax); l <= lmax; l++) {
          const double kz = 2.0 * M_PI * l * lzr;
          const double q2 = kx * kx + ky * ky + kz * kz;
          if (q2 < kc2) {
            kv.push_back(make_double3(kx, ky, kz));
            ksq.push_back(q2);
            const double bb = 1.0 / q2 * std::exp(-q2 * a2r / 4.0);
            bk.push_back(bb);
            ak.push_back(8.0 * M_PI * Vr * bb);
          }
        }
      }
    }
    const int nk = (int)kv.size();
    if (nk == 0 || b.natoms == 0) continue;
    Allocs kt;
    double3 *d_kv = kt.get<double3>(nk);
    double *d_a = kt.get<double>(nk), *d_S = kt.get<double>(nk), *d_C = kt.get<double>(nk);
    if (!d_kv || !d_a || !d_S || !d_C) return fail(PMB_ERR_CUDA, "cudaMalloc failed for the Ewald sum");
    CK(cudaMemcpyAsync(d_kv, kv.data(), sizeof(double3) * nk, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_a, ak.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    if (ewald_recip_launch(s->d_pos, s->d_charge, b.atom0, b.natoms, d_kv, d_a, nk, d_S, d_C, d_f, st))
      return fail(PMB_ERR_CUDA, "Ewald kernels");
    std::vector<double> S(nk), Cc(nk);
    CK(cudaMemcpyAsync(S.data(), d_S, sizeof(double) * nk, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(Cc.data(), d_C, sizeof(double) * nk, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hf.data() + 3 * (size_t)b.atom0, d_f + 3 * (size_t)b.atom0, sizeof(double) * 3 * b.natoms,
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // energy and virial in the reference's k order (NonbondedFullEwaldSystemForce.h:1031-1083)
    double energy = 0, vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
    for (int k = 0; k < nk; k++) {
      const double e = bk[k] * (S[k] * S[k] + Cc[k] * Cc[k]);
      energy += e;
      const double c = 2.0 * (1.0 / ksq[k] + fac);
      const double3 q = kv[k];
      vxx += e * (1.0 - c * q.x * q.x);
      vxy -= e * c * q.x * q.y;
      vxz -= e * c * q.x * q.z;
      vyy += e * (1.0 - c * q.y * q.y);
      vyz -= e * c * q.y * q.z;
      vzz += e * (1.0 - c * q.z * q.z);
    }
    const double c = 4.0 * M_PI * Vr;
    if (energies) {
      double *eb = energies + (size_t)bi * PMB_E_STRIDE;
      eb[PMB_E_COULOMB] += c * energy;
      if (virial) {
        const double vv[9] = {vxx, vxy, vxz, vxy, vyy, vyz, vxz, vyz, vzz};
        for (int k = 0; k < 9; k++) eb[PMB_E_VIRIAL + k] += c * vv[k];
      }
    }
  }
  if (forces)
    for (size_t i = 0; i < hf.size(); i++) forces[i] += hf[i];
  return PMB_OK;
}

int pmb_vacuum_box(const double *pos, int n_atoms, double margin, double edges[3]) {
  if (!pos || !edges || n_atoms <= 0 || !(margin >= 0)) return fail(PMB_ERR_ARG, "positions, atom count, margin >= 0");
  for (int c = 0; c < 3; c++) {
    double lo = pos[c], hi = pos[c];
    for (int i = 1; i < n_atoms; i++) {
      lo = std::min(lo, pos[3 * i + c]);
      hi = std::max(hi, pos[3 * i + c]);
    }
    if (!std::isfinite(lo) || !std::isfinite(hi)) return fail(PMB_ERR_NUMERIC, "non-finite position");
    edges[c] = 2.0 * (hi - lo + margin) + 1.0;
  }
  return PMB_OK;
}

int pmb_system_set_vacuum(pmb_system *s, int on) {
  if (!s) return fail(PMB_ERR_ARG, "null system");
  s->vacuum = on != 0;
  if (s->nb_ready) {
    const unsigned v = s->vacuum ? 1u : 0u;
    CK(cudaMemcpyAsync(s->nb.ctl + 10, &v, sizeof(v), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  return PMB_OK;
}

int pmb_evaluate(pmb_system *s, pmb_force *const *fs, int n, const double *pos, double *forces,
                 double *energies, int virial) {
  using clk = std::chrono::steady_clock;
  const clk::time_point t0 = clk::now();
  if (!s || !pos) return fail(PMB_ERR_ARG, "null argument");
  if (s->vacuum) {
    // the periodic box stands in for vacuum only while no two atoms of a box are half an edge
    // apart: then every minimal-image difference is the plain difference
    for (const BoxDev &b : s->hbox)
      for (int c = 0; c < 3; c++) {
        double lo = pos[3 * b.atom0 + c], hi = lo;
        for (int i = b.atom0 + 1; i < b.atom0 + b.natoms; i++) {
          lo = std::min(lo, pos[3 * i + c]);
          hi = std::max(hi, pos[3 * i + c]);
        }
        if (!(hi - lo < 0.5 * b.L[c]))
          return fail(PMB_ERR_STATE, "vacuum: the atoms spread over half a box edge; make the system "
                                     "again with edges from pmb_vacuum_box");
      }
  }
  cudaStream_t st = s->stream;
  if (!s->ev_out[0])
    for (cudaEvent_t &e : s->ev_out) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  const long long nf = 3LL * s->natoms;
  const long long chunk = (nf + pmb_system::EVAL_CHUNKS - 1) / pmb_system::EVAL_CHUNKS;
  // a captured graph per force set, except under the stage profiler or on the legacy stream
  const bool graphed = s->eval_graph && !s->prof && st != nullptr && st != cudaStreamLegacy;
  // page-locked force array: added to on the device and copied back into directly
  // (asked of the driver at every call: an array freed and another allocated at its address may
  // differ, and a graph's copies must only ever run on page-locked memory)
  const bool direct = graphed && forces && nf > 0 && host_pinned(forces, nf);
  // page-locked positions as well: every copy is a node of the evaluation's graph (one launch)
  const bool embed = direct && host_pinned(pos, nf);
  if (direct && !s->copy) {  // (the copy stream last: a failure part-way is taken up again here)
    if (!s->d_fin) s->d_fin = s->a.get<double>((size_t)nf, false);  // freed with the system
    if (!s->d_fin) return fail(PMB_ERR_CUDA, "cudaMalloc failed for the force upload");
    if (!s->ev_pos) CK(cudaEventCreateWithFlags(&s->ev_pos, cudaEventDisableTiming));
    if (!s->ev_fin) CK(cudaEventCreateWithFlags(&s->ev_fin, cudaEventDisableTiming));
    CK(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking));
  }
  for (int attempt = 0; attempt < 3; attempt++) {
    if (!embed) CK(cudaMemcpyAsync(s->d_pos, pos, sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    s->have_pos = true;
    if (direct && !embed && attempt == 0) {
      // after the positions (the two uploads would share the link), beside the force kernels;
      // a retry keeps this copy of the caller's forces
      CK(cudaEventRecord(s->ev_pos, st));
      CK(cudaStreamWaitEvent(s->copy, s->ev_pos, 0));
      CK(cudaMemcpyAsync(s->d_fin, forces, sizeof(double) * nf, cudaMemcpyHostToDevice, s->copy));
      CK(cudaEventRecord(s->ev_fin, s->copy));
    }
    int rc;
    if (graphed) {
      rc = eval_graph_launch(s, fs, n, virial, direct, embed ? pos : nullptr, embed ? forces : nullptr);
      if (!rc && direct && !embed) {
        CK(cudaMemcpyAsync(forces, s->d_fout, sizeof(double) * nf, cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(s->ev_out[1], st));
      }
    } else {
      rc = pmb_evaluate_device(s, fs, n, nullptr, s->d_fout, s->d_eout, virial);
      if (!rc) rc = enqueue_eval_copies(s);
    }
    if (rc) {  // no copy from the caller's arrays is left in flight
      cudaStreamSynchronize(st);
      if (s->copy) cudaStreamSynchronize(s->copy);
      return rc;
    }
    const clk::time_point t1 = clk::now();
    CK(cudaEventSynchronize(s->ev_out[0]));
    const clk::time_point t2 = clk::now();
    rc = s->nb_ready && s->last_used_list ? status_code(s) : PMB_OK;
    if (rc == PMB_OK && !s->last_used_list)  // no list kernel looked at the positions
      for (long long i = 0; i < nf; i++)
        if (!std::isfinite(pos[i])) {
          rc = fail(PMB_ERR_NUMERIC, "non-finite position");
          break;
        }
    if (rc) {
      CK(cudaStreamSynchronize(st));  // the copies in flight land before a retry or return
      if (direct) {  // the caller's array gets its own values back
        CK(cudaMemcpyAsync(forces, s->d_fin, sizeof(double) * nf, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
      }
    }
    if (rc == PMB_ERR_CAPACITY) {
      if (grow_and_retry_needed(s)) return PMB_ERR_CUDA;
      continue;
    }
    if (rc) return rc;
    if (direct) {
      CK(cudaEventSynchronize(s->ev_out[1]));
    } else if (forces && nf >= (1 << 16)) {
      // large systems: the pool's threads share every piece as it lands
      if (!s->add_pool) {
        const unsigned hw = std::thread::hardware_concurrency();
        int dev = 0;
        CK(cudaGetDevice(&dev));
        s->add_pool = new AddPool();
        s->add_pool->start((int)std::max(1u, std::min(4u, hw / 4)), dev);
      }
      s->add_pool->run(forces, s->h_fout, nf, chunk, pmb_system::EVAL_CHUNKS, s->ev_out + 1);
    } else {
      for (int c = 0; c < pmb_system::EVAL_CHUNKS; c++) {
        CK(cudaEventSynchronize(s->ev_out[c + 1]));
        if (!forces) continue;
        const long long b0 = c * chunk, b1 = std::min(nf, b0 + chunk);
        double *__restrict__ dst = forces;
        const double *__restrict__ src = s->h_fout;
        for (long long i = b0; i < b1; i++) dst[i] += src[i];
      }
    }
    const clk::time_point t3 = clk::now();
    s->eval_ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    s->eval_ms[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
    s->eval_ms[2] = std::chrono::duration<double, std::milli>(t3 - t2).count();
    if (energies) {
      add_const(fs, n, s->nbox, virial, s->h_eout);
      for (int b = 0; b < s->nbox; b++) {
        for (int k = 0; k < E_VIR; k++) energies[b * PMB_E_STRIDE + k] += s->h_eout[b * ACC_PER_BOX + k];
        if (virial)
          for (int k = 0; k < 9; k++)
            energies[b * PMB_E_STRIDE + PMB_E_VIRIAL + k] += s->h_eout[b * ACC_PER_BOX + E_VIR + k];
      }
    }
    return PMB_OK;
  }
  return fail(PMB_ERR_CAPACITY, "neighbour list capacity exceeded after retries");
}

int pmb_force_evaluate(pmb_force *f, const double *pos, double *forces, double *energies, int virial) {
  if (!f) return fail(PMB_ERR_ARG, "null force");
  return pmb_evaluate(f->sys, &f, 1, pos, forces, energies, virial);
}

int pmb_profile(pmb_system *s, const double *pos, pmb_force *const *fs, int n, int nrep, int flush_l2,
                double *stage_ms, int max_stages, int *n_stages, char *names, int names_len) {
  if (!s || (n > 0 && !fs) || nrep < 1 || !stage_ms || !n_stages)
    return fail(PMB_ERR_ARG, "null argument");
  cudaStream_t st = s->stream;
  if (pos) {
    CK(cudaMemcpyAsync(s->d_pos, pos, sizeof(double) * 3 * s->natoms, cudaMemcpyHostToDevice, st));
    s->have_pos = true;
  }
  if (!s->have_pos) return fail(PMB_ERR_STATE, "no positions on the device yet: pass positions");
  const size_t flush_bytes = 256ull << 20;  // twice the 126 MB L2
  if (flush_l2 && !s->flush_buf) CK(cudaMalloc(&s->flush_buf, flush_bytes));
  SystemDev sd = s->dev();
  zero_accumulators(sd, st);
  int rc = enqueue_forces(s, fs, n, 0);  // warm-up (also sizes the neighbour list)
  if (rc) return rc;
  CK(cudaStreamSynchronize(st));
  std::vector<std::string> order;
  std::vector<double> acc;
  for (int r = 0; r < nrep; r++) {
    if (flush_l2) CK(cudaMemsetAsync(s->flush_buf, r & 0xff, flush_bytes, st));
    zero_accumulators(sd, st);
    std::vector<std::pair<std::string, cudaEvent_t>> ev;
    s->prof = &ev;
    mark(s, "start");
    rc = enqueue_forces(s, fs, n, 0);
    s->prof = nullptr;
    cudaStreamSynchronize(st);
    for (size_t i = 1; i < ev.size() && rc == 0; i++) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[i - 1].second, ev[i].second);
      auto it = std::find(order.begin(), order.end(), ev[i].first);
      if (it == order.end()) {
        order.push_back(ev[i].first);
        acc.push_back(ms);
      } else {
        acc[it - order.begin()] += ms;
      }
    }
    for (auto &e : ev) cudaEventDestroy(e.second);
    if (rc) return rc;
  }
  *n_stages = (int)std::min<size_t>(order.size(), (size_t)max_stages);
  std::string joined;
  for (int i = 0; i < *n_stages; i++) {
    stage_ms[i] = acc[i] / nrep;
    joined += (i ? "," : "") + order[i];
  }
  if (names && names_len > 0) {
    std::strncpy(names, joined.c_str(), (size_t)names_len - 1);
    names[names_len - 1] = 0;
  }
  CK(cudaGetLastError());
  return check_status(s);
}

int pmb_fp32_peak(double *tflops) {
  if (!tflops) return fail(PMB_ERR_ARG, "null argument");
  if (pmb_device_count() <= 0) return fail(PMB_ERR_CUDA, "no CUDA device");
  if (fp32_peak_probe(tflops)) return fail(PMB_ERR_CUDA, "FMA probe failed");
  return PMB_OK;
}

}  // extern "C"

// ======================================================================================== MD
struct pmb_md {
  pmb_system *sys = nullptr;
  std::vector<pmb_force *> forces;
  pmb_integrator_desc d{};
  IntegratorDev in{};
  Allocs a;
  double *d_vel = nullptr, *d_kin = nullptr;
  long long *d_step = nullptr;
  unsigned long long *d_box_seed = nullptr;  // per box noise seed and step offset
  long long *d_box_step0 = nullptr;
  std::vector<unsigned long long> h_box_seed;
  std::vector<long long> h_box_step0;
  bool have_state = false, use_graph = true;
  bool virial = false;  // the steps evaluate the virial (forces and RATTLE's constraint terms)
  long long steps = 0;  // steps since the state was set (a checkpoint's step count)
  cudaGraphExec_t g_first = nullptr, g_next = nullptr;
  long long graph_gen = -1;  // list generation the graphs were captured with
  int kernels_per_step = 0;
  std::vector<double> h_e, h_k;
  // SHAKE after every drift, RATTLE after every step (absent: ngroup == 0)
  ConstraintDev con{};
  bool shake = false, rattle = false;
  Allocs *con_a = nullptr;
  void drop_graphs() {
    if (g_first) cudaGraphExecDestroy(g_first);
    if (g_next) cudaGraphExecDestroy(g_next);
    g_first = g_next = nullptr;
  }
  ~pmb_md() {
    drop_graphs();
    delete con_a;
  }
};

namespace {

// One step of LeapfrogIntegrator::run: kick (the opening half kick for kick = 0.5), drift, and
// the step's forces.  With constraints, as the reference's modifier hooks place them
// (LeapfrogIntegrator.cpp:56-87): a full kick becomes half kick, RATTLE, half kick when RATTLE
// is on, and SHAKE follows every drift.
int md_step_enqueue(pmb_md *m, double kick) {
  pmb_system *s = m->sys;
  SystemDev sd = s->dev();
  if (kick == 1.0 && m->rattle) {
    integrate_half_kick(sd, m->in, s->stream);
    if (constraints_apply(m->con, m->in, 1, s->stream)) return fail(PMB_ERR_CUDA, "RATTLE launch");
    integrate_kick_drift(sd, m->in, 0.5, s->stream);
  } else {
    integrate_kick_drift(sd, m->in, kick, s->stream);
  }
  if (m->shake && constraints_apply(m->con, m->in, 0, s->stream)) return fail(PMB_ERR_CUDA, "SHAKE launch");
  return enqueue_forces(s, m->forces.data(), (int)m->forces.size(), m->virial ? 1 : 0);
}

// Before a capture: the list storage the run's forces need exists, and a change of list radius
// has been marked (a rebuild) outside the graph, so that the captured step neither allocates nor
// forces a rebuild on every replay.
int md_prepare_list(pmb_md *m) {
  pmb_system *s = m->sys;
  const double rlist = list_radius(s, m->forces.data(), (int)m->forces.size());
  if (rlist <= 0.0) return PMB_OK;
  int rc = ensure_nblist(s, rlist);
  if (rc) return rc;
  if (rlist != s->nb_build_rl) {
    CK(cudaMemsetAsync(s->nb.ctl + 3, 1, 1, s->stream));
    s->nb_build_rl = rlist;
  }
  return PMB_OK;
}

int md_capture(pmb_md *m, double kick, cudaGraphExec_t *out) {
  pmb_system *s = m->sys;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  int rc = md_step_enqueue(m, kick);
  cudaError_t e = cudaStreamEndCapture(s->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(PMB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  size_t nn = 0;
  if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
    std::vector<cudaGraphNode_t> nodes(nn);
    int kern = 0;
    if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
      for (auto nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) kern++;
      }
    m->kernels_per_step = kern;
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(PMB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  return PMB_OK;
}

}  // namespace

extern "C" {

pmb_md *pmb_md_create(pmb_system *s, pmb_force *const *fs, int n, const pmb_integrator_desc *d) {
  if (!s || !d || n < 0 || (n > 0 && !fs)) return fail(PMB_ERR_ARG, "null argument"), nullptr;
  if (d->kind != PMB_LEAPFROG && d->kind != PMB_LANGEVIN) return fail(PMB_ERR_ARG, "integrator kind"), nullptr;
  if (!(d->timestep_fs > 0)) return fail(PMB_ERR_ARG, "timestep > 0"), nullptr;
  if (d->kind == PMB_LANGEVIN && !(d->gamma_ps > 0 && d->temperature >= 0))
    return fail(PMB_ERR_ARG, "Langevin needs gamma > 0 and temperature >= 0"), nullptr;
  pmb_md *m = new pmb_md();
  m->sys = s;
  m->d = *d;
  for (int i = 0; i < n; i++) {
    if (!fs[i] || fs[i]->sys != s) {
      delete m;
      return fail(PMB_ERR_ARG, "force belongs to another system"), nullptr;
    }
    m->forces.push_back(fs[i]);
  }
  const double INV_TIMEFACTOR = 0.02045482828087295, BOLTZMANN = 0.001987191;
  m->d_vel = m->a.get<double>(3 * (size_t)s->natoms);
  m->d_kin = m->a.get<double>(s->nbox);
  m->d_step = m->a.get<long long>(1);
  m->h_box_seed.resize(s->nbox);
  m->h_box_step0.assign(s->nbox, 0);
  for (int b = 0; b < s->nbox; b++) m->h_box_seed[b] = d->seed + (unsigned long long)b;
  if (!m->d_vel || !m->d_kin || !m->d_step || upload(m->a, m->d_box_seed, m->h_box_seed) ||
      upload(m->a, m->d_box_step0, m->h_box_step0)) {
    delete m;
    return fail(PMB_ERR_CUDA, "allocation failed"), nullptr;
  }
  m->in.kind = d->kind;
  m->in.h = d->timestep_fs * INV_TIMEFACTOR;
  m->in.gamma = d->gamma_ps / (1000 * INV_TIMEFACTOR);  // LangevinLeapfrogIntegrator.cpp:28
  m->in.kT = BOLTZMANN * d->temperature;
  m->in.seed = d->seed;
  m->in.box_seed = m->d_box_seed;
  m->in.box_step0 = m->d_box_step0;
  m->in.mass = s->d_mass;
  m->in.pos = s->d_pos;
  m->in.vel = m->d_vel;
  m->in.step = m->d_step;
  m->h_e.assign((size_t)s->nbox * ACC_PER_BOX, 0.0);
  m->h_k.assign(s->nbox, 0.0);
  return m;
}

int pmb_md_destroy(pmb_md *m) {
  if (m) {
    cudaDeviceSynchronize();
    delete m;
  }
  return PMB_OK;
}

int pmb_md_use_graph(pmb_md *m, int enable) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  m->use_graph = enable != 0;
  return PMB_OK;
}

int pmb_md_kernels_per_step(pmb_md *m, int *n) {
  if (!m || !n) return fail(PMB_ERR_ARG, "null argument");
  *n = m->kernels_per_step;
  return PMB_OK;
}


int pmb_md_set_constraints(pmb_md *m, const pmb_constraint_desc *d) {
  if (!m || !d) return fail(PMB_ERR_ARG, "null argument");
  pmb_system *s = m->sys;
  const int nc = d->n_constraints;
  if (nc < 0 || (nc > 0 && (!d->atom1 || !d->atom2 || !d->rest_length)))
    return fail(PMB_ERR_ARG, "constraint arrays");
  // ModifierModule::addModifiers: a modifier is added only with epsilon > 0 and max_iter > 0
  const bool shake = d->shake && d->shake_epsilon > 0 && d->shake_max_iter > 0 && nc > 0;
  const bool rattle = d->rattle && d->rattle_epsilon > 0 && d->rattle_max_iter > 0 && nc > 0;
  if ((shake && d->shake_max_iter >= CON_MAX_SWEEPS) || (rattle && d->rattle_max_iter >= CON_MAX_SWEEPS))
    return fail(PMB_ERR_ARG, "max_iter must be below 256");
  for (int k = 0; k < nc; k++) {
    const int a = d->atom1[k], b = d->atom2[k];
    if (a < 0 || b < 0 || a >= s->natoms || b >= s->natoms || a == b)
      return fail(PMB_ERR_ARG, "constraint atom out of range");
    if (!(d->rest_length[k] > 0) || !std::isfinite(d->rest_length[k]))
      return fail(PMB_ERR_ARG, "constraint rest length must be positive");
  }
  // groups: connected components of the constraint graph (union-find), constraints of a group in
  // list order, atoms in order of first use
  std::vector<int> parent(s->natoms);
  for (int i = 0; i < s->natoms; i++) parent[i] = i;
  auto find = [&](int x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  for (int k = 0; k < nc; k++) {
    int ra = find(d->atom1[k]), rb = find(d->atom2[k]);
    if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
  }
  std::vector<int> gid(s->natoms, -1), group_of_con(nc);
  int ng = 0;
  for (int k = 0; k < nc; k++) {
    int r = find(d->atom1[k]);
    if (gid[r] < 0) gid[r] = ng++;
    group_of_con[k] = gid[r];
  }
  std::vector<std::vector<int>> gcons(ng), gatoms(ng);
  for (int k = 0; k < nc; k++) gcons[group_of_con[k]].push_back(k);
  std::vector<int> group_con(ng + 1, 0), group_atom(ng + 1, 0), atoms;
  std::vector<int2> local;
  std::vector<double> len;
  int max_atoms = 0, max_cons = 0;
  for (int g = 0; g < ng; g++) {
    std::vector<int> &ga = gatoms[g];
    auto local_of = [&](int a) {
      for (size_t i = 0; i < ga.size(); i++)
        if (ga[i] == a) return (int)i;
      ga.push_back(a);
      return (int)ga.size() - 1;
    };
    for (int k : gcons[g]) {
      const int la = local_of(d->atom1[k]), lb = local_of(d->atom2[k]);
      local.push_back(make_int2(la, lb));
      len.push_back(d->rest_length[k]);
    }
    if ((int)ga.size() > CON_MAX_ATOMS || (int)gcons[g].size() > CON_MAX_CONS)
      return fail(PMB_ERR_UNSUPPORTED, "a constrained group has more than 8 atoms or 16 constraints");
    max_atoms = std::max(max_atoms, (int)ga.size());
    max_cons = std::max(max_cons, (int)gcons[g].size());
    atoms.insert(atoms.end(), ga.begin(), ga.end());
    group_con[g + 1] = group_con[g] + (int)gcons[g].size();
    group_atom[g + 1] = (int)atoms.size();
  }
  CK(cudaStreamSynchronize(s->stream));
  m->drop_graphs();
  delete m->con_a;
  m->con_a = nullptr;
  m->con = ConstraintDev{};
  m->shake = shake;
  m->rattle = rattle;
  if (!shake && !rattle) return PMB_OK;
  Allocs *a = m->con_a = new Allocs();
  ConstraintDev &c = m->con;
  int *d_gc = nullptr, *d_ga = nullptr, *d_atoms = nullptr;
  int2 *d_local = nullptr;
  double *d_len = nullptr;
  if (upload(*a, d_gc, group_con) || upload(*a, d_ga, group_atom) || upload(*a, d_atoms, atoms) ||
      upload(*a, d_local, local) || upload(*a, d_len, len))
    return PMB_ERR_CUDA;
  c.rab = a->get<double>(3 * (size_t)nc);
  c.err = a->get<long long>(2 * (size_t)CON_ERR_BLOCK);
  c.sweeps = a->get<int>(2);
  c.win = a->get<double>((size_t)CON_WINDOW * 6 * max_atoms * ng, false);
  if (!c.rab || !c.err || !c.sweeps || !c.win) return fail(PMB_ERR_CUDA, "cudaMalloc failed for the constraints");
  // the first application scans every sweep up to the cap
  const int first[2] = {shake ? d->shake_max_iter : 0, rattle ? d->rattle_max_iter : 0};
  CK(cudaMemcpy(c.sweeps, first, sizeof(first), cudaMemcpyHostToDevice));
  c.ngroup = ng;
  c.ncons = nc;
  c.max_atoms = max_atoms;
  c.max_cons = max_cons;
  c.group_con = d_gc;
  c.group_atom = d_ga;
  c.atoms = d_atoms;
  c.con_local = d_local;
  c.len = d_len;
  // a group error above this is clamped in the sums (ng * clamp * 2^40 stays below 2^62); such a
  // sum already exceeds any epsilon below clamp / n_constraints
  c.clamp = std::min(1e6, 4611686018427387904.0 / (CON_ERR_SCALE * std::max(ng, 1)));
  const double TIMEFACTOR = 48.88821290839616;  // base/PMConstants.cpp:53
  c.dt = m->d.timestep_fs / TIMEFACTOR;  // ModifierShake.cpp:22, ModifierRattle.cpp:22
  c.virial = m->virial ? 1 : 0;
  c.eacc = s->d_eacc;
  c.atom_box = s->d_atom_box;
  c.shake_eps = d->shake_epsilon;
  c.shake_max = shake ? d->shake_max_iter : 0;
  c.rattle_eps = d->rattle_epsilon;
  c.rattle_max = rattle ? d->rattle_max_iter : 0;
  if (m->have_state) constraints_init(c, m->in, s->stream);
  CK(cudaGetLastError());
  return PMB_OK;
}

}  // extern "C"

namespace pmb {
int md_frame_source(pmb_md *m, const double **d_pos, int *n_atoms, cudaStream_t *stream, int *device) {
  if (!m->have_state) return fail(PMB_ERR_STATE, "pmb_md_set_state must come first");
  *d_pos = m->sys->d_pos;
  *n_atoms = m->sys->natoms;
  *stream = m->sys->stream;
  CK(cudaGetDevice(device));
  return PMB_OK;
}

int md_force_frame(pmb_md *m, double *d_out) {
  if (!m->have_state) return fail(PMB_ERR_STATE, "pmb_md_set_state must come first");
  pmb_system *s = m->sys;
  forces_to_double(s->dev(), d_out, s->stream);
  CK(cudaGetLastError());
  return PMB_OK;
}

int md_noise(pmb_md *m, int *kind, unsigned long long *seed, long long *steps) {
  *kind = m->d.kind;
  *seed = m->h_box_seed[0];
  *steps = m->h_box_step0[0] + m->steps;
  return PMB_OK;
}
}  // namespace pmb

extern "C" {

int pmb_md_constraint_sweeps(pmb_md *m, int *shake_sweeps, int *rattle_sweeps) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  int h[2] = {0, 0};
  if (m->con.sweeps) {
    CK(cudaMemcpyAsync(h, m->con.sweeps, sizeof(h), cudaMemcpyDeviceToHost, m->sys->stream));
    CK(cudaStreamSynchronize(m->sys->stream));
  }
  if (shake_sweeps) *shake_sweeps = h[0];
  if (rattle_sweeps) *rattle_sweeps = h[1];
  return PMB_OK;
}

int pmb_md_set_state(pmb_md *m, const double *pos, const double *vel) {
  return pmb_md_set_checkpoint(m, pos, vel, nullptr, 0);
}

int pmb_md_get_checkpoint(pmb_md *m, double *pos, double *vel, double *list_reference, long long *step) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  if (!m->have_state) return fail(PMB_ERR_STATE, "pmb_md_set_state must come first");
  pmb_system *s = m->sys;
  const size_t bytes = sizeof(double) * 3 * (size_t)s->natoms;
  if (pos) CK(cudaMemcpyAsync(pos, s->d_pos, bytes, cudaMemcpyDeviceToHost, s->stream));
  if (vel) CK(cudaMemcpyAsync(vel, m->d_vel, bytes, cudaMemcpyDeviceToHost, s->stream));
  // the list's reference positions (those of its last build); a run without a list has none,
  // and its positions stand in
  if (list_reference)
    CK(cudaMemcpyAsync(list_reference, s->nb_ready ? s->nb.xref : s->d_pos, bytes, cudaMemcpyDeviceToHost,
                       s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (step) *step = m->steps;
  return check_status(s);
}

int pmb_md_set_checkpoint(pmb_md *m, const double *pos, const double *vel, const double *list_reference,
                          long long step) {
  if (!m || !pos) return fail(PMB_ERR_ARG, "null argument");
  if (step < 0) return fail(PMB_ERR_ARG, "step count < 0");
  pmb_system *s = m->sys;
  for (int i = 0; i < 3 * s->natoms; i++)
    if (!std::isfinite(pos[i]) || (vel && !std::isfinite(vel[i])) ||
        (list_reference && !std::isfinite(list_reference[i])))
      return fail(PMB_ERR_NUMERIC, "non-finite state");
  const size_t bytes = sizeof(double) * 3 * (size_t)s->natoms;
  SystemDev sd = s->dev();
  m->have_state = false;
  for (int attempt = 0; attempt < 3; attempt++) {
    int rc = PMB_OK;
    if (list_reference) {
      // the list of the run the checkpoint comes from: built at its reference positions (the
      // build is deterministic), so that every later step sums the same tiles in the same order
      CK(cudaMemcpyAsync(s->d_pos, list_reference, bytes, cudaMemcpyHostToDevice, s->stream));
      s->have_pos = true;
      if (s->nb_ready) CK(cudaMemsetAsync(s->nb.ctl + 3, 1, 1, s->stream));  // rebuild
      zero_accumulators(sd, s->stream);
      rc = enqueue_forces(s, m->forces.data(), (int)m->forces.size(), m->virial ? 1 : 0);
      if (rc) return rc;
      rc = check_status(s);
    }
    if (rc == PMB_OK) {
      CK(cudaMemcpyAsync(s->d_pos, pos, bytes, cudaMemcpyHostToDevice, s->stream));
      s->have_pos = true;
      if (vel) CK(cudaMemcpyAsync(m->d_vel, vel, bytes, cudaMemcpyHostToDevice, s->stream));
      else CK(cudaMemsetAsync(m->d_vel, 0, bytes, s->stream));
      // the Langevin noise counter: the restored run draws the streams the original would have
      CK(cudaMemcpyAsync(m->d_step, &step, sizeof(long long), cudaMemcpyHostToDevice, s->stream));
      constraints_init(m->con, m->in, s->stream);  // the new positions are SHAKE's last ones
      zero_accumulators(sd, s->stream);
      rc = enqueue_forces(s, m->forces.data(), (int)m->forces.size(), m->virial ? 1 : 0);
      if (rc) return rc;
      rc = check_status(s);  // also waits for the step count's host copy
    }
    if (rc == PMB_ERR_CAPACITY) {
      if (grow_and_retry_needed(s)) return PMB_ERR_CUDA;
      m->drop_graphs();  // they hold the old list's buffers
      continue;
    }
    if (rc) return rc;
    m->have_state = true;
    m->steps = step;
    return PMB_OK;
  }
  return fail(PMB_ERR_CAPACITY, "neighbour list capacity exceeded");
}

int pmb_md_set_box_noise(pmb_md *m, const unsigned long long *seeds, const long long *steps) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  pmb_system *s = m->sys;
  if (steps)
    for (int b = 0; b < s->nbox; b++)
      if (steps[b] < 0) return fail(PMB_ERR_ARG, "step count < 0");
  for (int b = 0; b < s->nbox; b++) {
    if (seeds) m->h_box_seed[b] = seeds[b];
    if (steps) m->h_box_step0[b] = steps[b] - m->steps;
  }
  CK(cudaMemcpyAsync(m->d_box_seed, m->h_box_seed.data(), sizeof(unsigned long long) * s->nbox,
                     cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(m->d_box_step0, m->h_box_step0.data(), sizeof(long long) * s->nbox,
                     cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return PMB_OK;
}

int pmb_md_get_box_noise(const pmb_md *m, unsigned long long *seeds, long long *steps) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  for (int b = 0; b < m->sys->nbox; b++) {
    if (seeds) seeds[b] = m->h_box_seed[b];
    if (steps) steps[b] = m->h_box_step0[b] + m->steps;
  }
  return PMB_OK;
}

int pmb_md_run(pmb_md *m, int n) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  if (!m->have_state) return fail(PMB_ERR_STATE, "pmb_md_set_state must come first");
  if (n < 1) return PMB_OK;
  pmb_system *s = m->sys;
  // the legacy default stream cannot be captured: replay eagerly there
  const bool graph_ok = s->stream != nullptr && s->stream != cudaStreamLegacy;
  if (m->use_graph && graph_ok) {
    int prc = md_prepare_list(m);
    if (prc) return prc;
    if (m->graph_gen != s->nb_gen) m->drop_graphs();
    m->graph_gen = s->nb_gen;
    if (!m->g_first) {
      int rc = md_capture(m, 0.5, &m->g_first);
      if (rc) return rc;
    }
    if (n > 1 && !m->g_next) {
      int rc = md_capture(m, 1.0, &m->g_next);
      if (rc) return rc;
    }
    CK(cudaGraphLaunch(m->g_first, s->stream));
    for (int i = 1; i < n; i++) CK(cudaGraphLaunch(m->g_next, s->stream));
  } else {
    int rc = md_step_enqueue(m, 0.5);
    if (rc) return rc;
    for (int i = 1; i < n; i++) {
      rc = md_step_enqueue(m, 1.0);
      if (rc) return rc;
    }
  }
  integrate_half_kick(s->dev(), m->in, s->stream);
  if (m->rattle && constraints_apply(m->con, m->in, 1, s->stream)) return fail(PMB_ERR_CUDA, "RATTLE launch");
  CK(cudaGetLastError());
  m->steps += n;
  return PMB_OK;
}

int pmb_md_set_virial(pmb_md *m, int on) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  pmb_system *s = m->sys;
  CK(cudaStreamSynchronize(s->stream));
  m->virial = on != 0;
  m->con.virial = m->virial ? 1 : 0;
  m->con.eacc = s->d_eacc;
  m->con.atom_box = s->d_atom_box;
  m->drop_graphs();  // the step's kernels differ
  return PMB_OK;
}

int pmb_md_time(pmb_md *m, int n, double *ms) {
  if (!m || !ms || n < 1) return fail(PMB_ERR_ARG, "md, n_steps >= 1 and an output");
  if (!m->have_state) return fail(PMB_ERR_STATE, "pmb_md_set_state must come first");
  pmb_system *s = m->sys;
  cudaEvent_t a = nullptr, b = nullptr;
  CK(cudaEventCreate(&a));
  if (cudaEventCreate(&b) != cudaSuccess) {
    cudaEventDestroy(a);
    return fail(PMB_ERR_CUDA, "cudaEventCreate");
  }
  int rc = PMB_OK;
  float t = 0.f;
  if (cudaEventRecord(a, s->stream) != cudaSuccess) rc = fail(PMB_ERR_CUDA, "cudaEventRecord");
  if (!rc) rc = pmb_md_run(m, n);
  if (!rc && (cudaEventRecord(b, s->stream) != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess ||
              cudaEventElapsedTime(&t, a, b) != cudaSuccess))
    rc = fail(PMB_ERR_CUDA, "timing events");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (!rc) rc = check_status(s);
  *ms = (double)t / n;
  return rc;
}

int pmb_md_device_bytes(const pmb_md *m, unsigned long long *bytes) {
  if (!m || !bytes) return fail(PMB_ERR_ARG, "null argument");
  const pmb_system *s = m->sys;
  size_t b = s->a.bytes + s->nba.bytes + m->a.bytes + (m->con_a ? m->con_a->bytes : 0) +
             (s->flush_buf ? (256ull << 20) : 0);
  for (const pmb_force *f : m->forces) b += f->a.bytes;
  *bytes = (unsigned long long)b;
  return PMB_OK;
}

int pmb_md_get_state(pmb_md *m, double *pos, double *vel) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  pmb_system *s = m->sys;
  if (pos) CK(cudaMemcpyAsync(pos, s->d_pos, sizeof(double) * 3 * s->natoms, cudaMemcpyDeviceToHost, s->stream));
  if (vel) CK(cudaMemcpyAsync(vel, m->d_vel, sizeof(double) * 3 * s->natoms, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return check_status(s);
}

int pmb_md_get_forces(pmb_md *m, double *forces) {
  if (!m || !forces) return fail(PMB_ERR_ARG, "null argument");
  pmb_system *s = m->sys;
  forces_to_double(s->dev(), s->d_fout, s->stream);
  CK(cudaMemcpyAsync(forces, s->d_fout, sizeof(double) * 3 * s->natoms, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return PMB_OK;
}

int pmb_md_energies(pmb_md *m, double *energies, double *kinetic) {
  if (!m) return fail(PMB_ERR_ARG, "null md");
  pmb_system *s = m->sys;
  SystemDev sd = s->dev();
  energies_to_double(sd, nullptr, s->d_eout, s->stream);
  kinetic_energy(sd, m->in, m->d_kin, s->stream);
  CK(cudaMemcpyAsync(m->h_e.data(), s->d_eout, sizeof(double) * m->h_e.size(), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(m->h_k.data(), m->d_kin, sizeof(double) * m->h_k.size(), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  add_const(m->forces.data(), (int)m->forces.size(), s->nbox, m->virial ? 1 : 0, m->h_e.data());
  for (int b = 0; b < s->nbox; b++) {
    if (energies)
      for (int k = 0; k < PMB_E_STRIDE; k++)
        energies[b * PMB_E_STRIDE + k] = k < E_VIR || (m->virial && k < E_VIR + 9) ? m->h_e[b * ACC_PER_BOX + k] : 0.0;
    if (kinetic) kinetic[b] = m->h_k[b];
  }
  return check_status(s);
}

}  // extern "C"

// Allocation-free NonbondedCutoff evaluation: the only scratch is the static energy/virial array
// of pmb_pair.cu; topology and LJ tables are the system's, created by pmb_system_create.
static_assert(STATIC_MAX_BOXES == PMB_STATIC_MAX_BOXES, "static scratch size mismatch");

extern "C" int pmb_cutoff_evaluate_static(pmb_force *f, const double *d_positions, double *d_forces,
                                          double *d_energies, int virial) {
  if (!f || !d_positions || !d_forces) return fail(PMB_ERR_ARG, "null argument");
  if (f->kind != PMB_FORCE_CUTOFF)
    return fail(PMB_ERR_UNSUPPORTED, "pmb_cutoff_evaluate_static evaluates NonbondedCutoff forces only");
  pmb_system *s = f->sys;
  if (s->nbox > PMB_STATIC_MAX_BOXES)
    return fail(PMB_ERR_CAPACITY, "pmb_cutoff_evaluate_static: " + std::to_string(s->nbox) +
                                      " boxes exceed its static scratch of PMB_STATIC_MAX_BOXES = " +
                                      std::to_string(PMB_STATIC_MAX_BOXES) + " boxes");
  long long *eacc = nullptr;
  CK(static_eacc_address(&eacc));
  // the cutoff branch of pair_jobs, without its host vector
  PairParams p = base_params(s, virial);
  p.do_lj = f->d.lj;
  p.coul_mode = f->d.coulomb ? 1 : 0;
  p.lj_sw = make_switch(f->d.lj_switch, f->d.lj_switchon, f->d.lj_cutoff);
  p.coul_sw = make_switch(f->d.coulomb_switch, f->d.coulomb_switchon, f->d.coulomb_cutoff);
  p.lj_cut2 = f->d.lj_cutoff * f->d.lj_cutoff;
  p.coul_cut2 = f->d.coulomb_cutoff * f->d.coulomb_cutoff;
  const double rc = force_pair_cutoff(f);
  p.cut2 = rc * rc;
  int max_box_atoms = 0;
  for (const BoxDev &b : s->hbox) max_box_atoms = std::max(max_box_atoms, b.natoms);
  SystemDev sd = s->dev();
  sd.eacc = eacc;
  sd.facc = nullptr;
  CK(pair_allpairs_launch(sd, p, s->d_lj, d_positions, d_forces, eacc, max_box_atoms, s->stream));
  if (d_energies) {
    energies_to_double(sd, nullptr, d_energies, s->stream);
    CK(cudaGetLastError());
  }
  return PMB_OK;
}
