// Trajectory output from device-resident MD state (host code).
//
// Files are the reference's formats byte for byte:
//   DCD as DCDTrajectoryWriter writes it (io/DCDTrajectoryWriter.cpp:75-233): a CHARMM-24 header
//   on the first frame (frame count at bytes 8 and 20, updated on every later frame), title
//   records "Remarks: ..." in 80-byte lines, then per frame three Fortran records of float32 x,
//   y and z; OutputDCDTrajectory passes timestep 1.0 (output/OutputDCDTrajectory.cpp:33), so
//   that is the default here as well.  The first title line names the file and the build, as the
//   reference's does (its bytes therefore differ between builds of either program).
//   XYZ as XYZWriter::write (io/XYZWriter.cpp:28-53): the atom count, then per atom the name, a
//   tab and the three coordinates in 24-wide fields at 15 significant digits; every frame
//   rewrites the file (final-position output).
//   XYZ trajectory as XYZTrajectoryWriter (io/XYZTrajectoryWriter.cpp:64-160): a first line with
//   the frame count in 19 characters (rewritten on every frame), then the frames in the XYZ form.
//   Checkpoints as OutputCheckpoint writes them (output/OutputCheckpoint.cpp:58-178): positions
//   and velocities in the XYZ form, then the checkpoint file of CheckpointConfigWriter.
//   Minimal-image DCD frames as OutputCache::getMinimalPositions makes them
//   (topology/SemiGenericTopology.h:127-150), computed by the writer thread on the host copy.
//
// pmb_md_write_frame takes a frame off the device without stopping it: a device-to-device
// snapshot of the positions on the system's stream (the next step waits only for that), the
// snapshot's copy into one of three pinned host buffers on the trajectory's own stream, and a
// writer thread per trajectory that waits for the copy and appends the frame.  The caller waits
// only when all three buffers are still in flight.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <iomanip>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "pmb200.h"
#include "pmb_internal.h"

namespace pmb {
// defined in pmb_api.cu: the positions, atom count and stream of an MD run
int md_frame_source(pmb_md *md, const double **d_pos, int *n_atoms, cudaStream_t *stream, int *device);
// enqueues the MD run's forces (of its last evaluation) as FP64 into d_out on its stream
int md_force_frame(pmb_md *md, double *d_out);
// the MD run's integrator kind and the noise stream of its first box (seed, steps drawn)
int md_noise(pmb_md *md, int *kind, unsigned long long *seed, long long *steps);
}  // namespace pmb

using namespace pmb;

namespace {

const double INV_TIMEFACTOR = 0.02045482828087295;  // base/PMConstants.cpp:54
constexpr int STAGES = 3;

bool host_little_endian() {
  const unsigned one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

template <typename T>
T swapped(T v) {
  unsigned char b[sizeof(T)];
  std::memcpy(b, &v, sizeof(T));
  for (size_t i = 0; i < sizeof(T) / 2; i++) std::swap(b[i], b[sizeof(T) - 1 - i]);
  std::memcpy(&v, b, sizeof(T));
  return v;
}

std::string right_fill(const std::string &s, size_t n) {
  return s.size() < n ? s + std::string(n - s.size(), ' ') : s.substr(0, n);
}

// One frame as XYZWriter::write / XYZTrajectoryWriter::write print it (io/XYZWriter.cpp:42-53).
std::string xyz_text(int n, const std::vector<std::string> &names, const double *v) {
  std::ostringstream o;
  o << n << std::endl;
  o.precision(15);
  for (int i = 0; i < n; i++) {
    o << names[i] << "\t";
    for (int c = 0; c < 3; c++) {
      o.width(24);
      o << v[3 * i + c];
    }
    o << std::endl;
  }
  return o.str();
}

bool write_file(const std::string &path, const std::string &text) {
  std::FILE *x = std::fopen(path.c_str(), "wb");
  if (!x) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), x) == text.size();
  return std::fclose(x) == 0 && ok;
}

// Minimal image of one frame (SemiGenericTopology::minimalImage with the orthogonal
// PeriodicBoundaryConditions of topology/PeriodicBoundaryConditions.cpp:32-77, .h:150-185).
struct MinimalImage {
  std::vector<std::vector<int>> atoms;                  // per molecule, ascending
  std::vector<std::vector<std::pair<int, int>>> pairs;  // per molecule, ascending (first < second)
  std::vector<double> mass;
  double L[3], Lr[3], origin[3], D;

  // the lattice translation of d (minimalTranslationDifference / Position): none while |d|^2 is
  // within the safe distance, else L rint(d / L) per axis
  void translation(const double d[3], double t[3]) const {
    if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] <= D) {
      t[0] = t[1] = t[2] = 0.0;
      return;
    }
    for (int c = 0; c < 3; c++) t[c] = L[c] * std::rint(Lr[c] * d[c]);
  }
  void apply(double *x) const {
    const double EPS = 1.0e-14;  // base/PMConstants.cpp:50
    for (size_t m = 0; m < atoms.size(); m++) {
      for (const std::pair<int, int> &p : pairs[m]) {
        const double d[3] = {x[3 * p.second] - x[3 * p.first], x[3 * p.second + 1] - x[3 * p.first + 1],
                             x[3 * p.second + 2] - x[3 * p.first + 2]};
        double t[3];
        translation(d, t);
        if (t[0] * t[0] + t[1] * t[1] + t[2] * t[2] > EPS)
          for (int c = 0; c < 3; c++) x[3 * p.second + c] -= t[c];
      }
      // molecularCenterOfMass (topology/TopologyUtilities.cpp:646-674): Kahan summation
      const std::vector<int> &a = atoms[m];
      double mt = mass[a[0]], cen[3], kc[3] = {0.0, 0.0, 0.0};
      for (int c = 0; c < 3; c++) cen[c] = x[3 * a[0] + c] * mt;
      for (size_t i = 1; i < a.size(); i++) {
        const double w = mass[a[i]];
        mt += w;
        for (int c = 0; c < 3; c++) {
          const double tx = x[3 * a[i] + c] * w, ty = tx - kc[c], tt = cen[c] + ty;
          kc[c] = (tt - cen[c]) - ty;
          cen[c] = tt;
        }
      }
      double d[3], t[3];
      for (int c = 0; c < 3; c++) d[c] = cen[c] / mt - origin[c];
      translation(d, t);
      if (t[0] * t[0] + t[1] * t[1] + t[2] * t[2] > EPS)
        for (int i : a)
          for (int c = 0; c < 3; c++) x[3 * i + c] -= t[c];
    }
  }
};

}  // namespace

struct pmb_traj {
  int kind = 0;  // 0 DCD, 1 XYZ, 2 XYZ trajectory
  std::string path, comment;
  int n_atoms = 0, first_step = 0;
  double timestep = 1.0;
  bool swap = false;
  std::vector<std::string> names;
  long frames = 0;
  std::FILE *f = nullptr;
  std::vector<float> fx, fy, fz;
  // asynchronous frames
  struct Stage {
    double *host = nullptr;       // pinned
    double *dev = nullptr;        // device snapshot of the positions
    cudaEvent_t taken = nullptr;  // snapshot done (system stream)
    cudaEvent_t ev = nullptr;     // host copy done (copy stream)
    bool busy = false;
  } stage[STAGES];
  cudaStream_t copy = nullptr;
  std::deque<int> queue;
  std::mutex mu;
  std::condition_variable cv;
  std::thread th;
  bool stop = false, started = false;
  int err = PMB_OK;
  std::string err_msg;
  int device = -1;  // the device of the first frame: the staging buffers and copy stream live there
  MinimalImage *minimal = nullptr;  // DCD frames in minimal image
  std::vector<double> scratch;      // a frame's minimal-image copy

  template <typename T>
  void put(T v) {
    if (swap) v = swapped(v);
    std::fwrite(&v, sizeof(T), 1, f);
  }

  int write_dcd(const double *pos) {
    const int n = n_atoms;
    if (frames == 0) {
      f = std::fopen(path.c_str(), "wb+");
      if (!f) return PMB_ERR_ARG;
      const int csize = (int)comment.size() + 9;  // 9 for "Remarks: "
      int n2 = (csize + 80) / 80;
      if (csize % 80 != 0) n2++;
      const float ts = (float)((double)(float)timestep * INV_TIMEFACTOR);
      put<int32_t>(84);
      std::fwrite("CORD", 1, 4, f);
      put<int32_t>(1);           // frames
      put<int32_t>(first_step);  // first step
      put<int32_t>(1);           // steps between frames
      put<int32_t>(1);           // frames again
      for (int i = 0; i < 5; i++) put<int32_t>(0);
      put<float>(ts);
      for (int i = 0; i < 9; i++) put<int32_t>(0);
      put<int32_t>(24);  // CHARMM version
      put<int32_t>(84);
      put<int32_t>(n2 * 80 + 4);
      put<int32_t>(n2);
      const std::string first = "Remarks: File '" + path + "'. protomol3_b200 (" + __DATE__ + " at " + __TIME__ + ")";
      std::fwrite(right_fill(first, 80).data(), 1, 80, f);
      const size_t nc = (size_t)(n2 - 1) * 80;
      std::fwrite(right_fill("Remarks: " + comment, nc).data(), 1, nc, f);
      put<int32_t>(n2 * 80 + 4);
      put<int32_t>(4);
      put<int32_t>(n);
      put<int32_t>(4);
    } else {
      const int32_t sets = (int32_t)(frames + 1);
      std::fseek(f, 8, SEEK_SET);
      put<int32_t>(sets);
      std::fseek(f, 20, SEEK_SET);
      put<int32_t>(sets);
      std::fseek(f, 0, SEEK_END);
    }
    fx.resize(n);
    fy.resize(n);
    fz.resize(n);
    for (int i = 0; i < n; i++) {
      fx[i] = (float)pos[3 * i];
      fy[i] = (float)pos[3 * i + 1];
      fz[i] = (float)pos[3 * i + 2];
      if (swap) {
        fx[i] = swapped(fx[i]);
        fy[i] = swapped(fy[i]);
        fz[i] = swapped(fz[i]);
      }
    }
    const int32_t rec = 4 * n;
    for (const std::vector<float> *c : {&fx, &fy, &fz}) {
      put<int32_t>(rec);
      std::fwrite(c->data(), sizeof(float), (size_t)n, f);
      put<int32_t>(rec);
    }
    std::fflush(f);
    frames++;
    return std::ferror(f) ? PMB_ERR_ARG : PMB_OK;
  }

  int write_xyz(const double *pos) {
    const bool ok = write_file(path, xyz_text(n_atoms, names, pos));
    frames++;
    return ok ? PMB_OK : PMB_ERR_ARG;
  }

  // XYZTrajectoryWriter::reopen + write: the frame count line, 19 characters and a newline,
  // rewritten in place; the frame appended
  int write_xyz_trajectory(const double *pos) {
    const std::string head = right_fill(std::to_string(frames + 1), 19) + "\n";
    std::FILE *x = std::fopen(path.c_str(), frames == 0 ? "wb" : "r+b");
    if (!x) return PMB_ERR_ARG;
    bool ok = std::fwrite(head.data(), 1, head.size(), x) == head.size();
    const std::string body = xyz_text(n_atoms, names, pos);
    ok = ok && std::fseek(x, 0, SEEK_END) == 0 && std::fwrite(body.data(), 1, body.size(), x) == body.size();
    ok = std::fclose(x) == 0 && ok;
    frames++;
    return ok ? PMB_OK : PMB_ERR_ARG;
  }

  int write(const double *pos) {
    if (kind == 1) return write_xyz(pos);
    if (kind == 2) return write_xyz_trajectory(pos);
    if (minimal) {
      scratch.assign(pos, pos + 3 * (size_t)n_atoms);
      minimal->apply(scratch.data());
      return write_dcd(scratch.data());
    }
    return write_dcd(pos);
  }

  void writer_loop() {
    if (device >= 0) cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      cv.wait(lk, [&] { return stop || !queue.empty(); });
      if (queue.empty()) return;
      const int k = queue.front();
      lk.unlock();
      int rc = PMB_OK;
      if (cudaEventSynchronize(stage[k].ev) != cudaSuccess) rc = PMB_ERR_CUDA;
      if (rc == PMB_OK) rc = write(stage[k].host);
      lk.lock();
      queue.pop_front();
      stage[k].busy = false;
      if (rc != PMB_OK && err == PMB_OK) {
        err = rc;
        err_msg = rc == PMB_ERR_CUDA ? "trajectory frame copy failed" : "cannot write " + path;
      }
      cv.notify_all();
    }
  }

  int flush() {
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] {
      if (!queue.empty()) return false;
      for (const Stage &s : stage)
        if (s.busy) return false;
      return true;
    });
    return err;
  }

  ~pmb_traj() {
    if (started) {
      flush();
      {
        std::lock_guard<std::mutex> lk(mu);
        stop = true;
      }
      cv.notify_all();
      th.join();
    }
    for (Stage &s : stage) {
      if (s.host) cudaFreeHost(s.host);
      if (s.dev) cudaFree(s.dev);
      if (s.taken) cudaEventDestroy(s.taken);
      if (s.ev) cudaEventDestroy(s.ev);
    }
    if (copy) cudaStreamDestroy(copy);
    if (f) std::fclose(f);
    delete minimal;
  }
};

extern "C" {

pmb_traj *pmb_traj_open_dcd(const char *path, int n_atoms, double timestep, int first_step, int little_endian,
                            const char *comment) {
  if (!path || !*path || n_atoms <= 0) return set_error("trajectory path and atom count"), nullptr;
  pmb_traj *t = new pmb_traj();
  t->kind = 0;
  t->path = path;
  t->n_atoms = n_atoms;
  t->timestep = timestep;
  t->first_step = first_step;
  t->swap = (little_endian != 0) != host_little_endian();
  t->comment = comment ? comment : "";
  return t;
}

pmb_traj *pmb_traj_open_xyz(const char *path, int n_atoms, const char *const *names) {
  if (!path || !*path || n_atoms <= 0 || !names) return set_error("trajectory path, atom count and names"), nullptr;
  pmb_traj *t = new pmb_traj();
  t->kind = 1;
  t->path = path;
  t->n_atoms = n_atoms;
  for (int i = 0; i < n_atoms; i++) {
    if (!names[i]) {
      delete t;
      return set_error("null atom name"), nullptr;
    }
    t->names.push_back(names[i]);
  }
  return t;
}

int pmb_traj_write_host(pmb_traj *t, const double *positions) {
  if (!t || !positions) return set_error("null argument"), PMB_ERR_ARG;
  int rc = t->flush();  // frames already queued go first
  if (rc) return set_error(t->err_msg), rc;
  rc = t->write(positions);
  if (rc) set_error("cannot write " + t->path);
  return rc;
}

}  // extern "C"

namespace {
// A frame of the MD run's positions (forces = false) or forces, taken without stopping the device.
int md_frame(pmb_md *md, pmb_traj *t, bool forces) {
  if (!md || !t) return set_error("null argument"), PMB_ERR_ARG;
  const double *d_pos = nullptr;
  int n = 0, dev = 0;
  cudaStream_t st = nullptr;
  int rc = md_frame_source(md, &d_pos, &n, &st, &dev);
  if (rc) return rc;
  if (n != t->n_atoms) return set_error("trajectory atom count differs from the MD run's"), PMB_ERR_ARG;
  // the staging buffers and the copy stream belong to the device of the first frame (also when
  // that attempt failed half way and this call retries it)
  if (t->device >= 0 && dev != t->device)
    return set_error("trajectory frames come from device " + std::to_string(t->device) +
                     "; this MD run is on device " + std::to_string(dev)),
           PMB_ERR_ARG;
  if (!t->started) {
    t->device = dev;
    const size_t bytes = sizeof(double) * 3 * (size_t)n;
    // what a failed attempt obtained is kept (and freed with the trajectory); a retry fills the rest
    if (!t->copy && cudaStreamCreateWithFlags(&t->copy, cudaStreamNonBlocking) != cudaSuccess)
      return set_error("copy stream for the trajectory"), PMB_ERR_CUDA;
    for (pmb_traj::Stage &s : t->stage) {
      if ((!s.host && cudaMallocHost(&s.host, bytes) != cudaSuccess) ||
          (!s.dev && cudaMalloc(&s.dev, bytes) != cudaSuccess) ||
          (!s.taken && cudaEventCreateWithFlags(&s.taken, cudaEventDisableTiming) != cudaSuccess) ||
          (!s.ev && cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming) != cudaSuccess))
        return set_error("staging buffers for the trajectory"), PMB_ERR_CUDA;
    }
    t->th = std::thread([t] { t->writer_loop(); });
    t->started = true;
  }
  int k = -1;
  {
    std::unique_lock<std::mutex> lk(t->mu);
    t->cv.wait(lk, [&] {
      for (int i = 0; i < STAGES; i++)
        if (!t->stage[i].busy) return true;
      return false;
    });
    if (t->err) return set_error(t->err_msg), t->err;
    for (int i = 0; i < STAGES && k < 0; i++)
      if (!t->stage[i].busy) k = i;
    t->stage[k].busy = true;
  }
  // a device snapshot on the run's stream (microseconds), then the host copy on the trajectory's
  // own stream, beside the steps that follow
  pmb_traj::Stage &sg = t->stage[k];
  const size_t bytes = sizeof(double) * 3 * (size_t)n;
  const bool snap = forces ? md_force_frame(md, sg.dev) == PMB_OK
                           : cudaMemcpyAsync(sg.dev, d_pos, bytes, cudaMemcpyDeviceToDevice, st) == cudaSuccess;
  if (!snap || cudaEventRecord(sg.taken, st) != cudaSuccess || cudaStreamWaitEvent(t->copy, sg.taken, 0) != cudaSuccess ||
      cudaMemcpyAsync(sg.host, sg.dev, bytes, cudaMemcpyDeviceToHost, t->copy) != cudaSuccess ||
      cudaEventRecord(sg.ev, t->copy) != cudaSuccess) {
    std::lock_guard<std::mutex> lk(t->mu);
    t->stage[k].busy = false;
    return set_error("trajectory frame copy"), PMB_ERR_CUDA;
  }
  {
    std::lock_guard<std::mutex> lk(t->mu);
    t->queue.push_back(k);
  }
  t->cv.notify_all();
  return PMB_OK;
}
}  // namespace

extern "C" {

int pmb_md_write_frame(pmb_md *md, pmb_traj *t) { return md_frame(md, t, false); }

int pmb_md_write_force_frame(pmb_md *md, pmb_traj *t) { return md_frame(md, t, true); }

pmb_traj *pmb_traj_open_xyz_trajectory(const char *path, int n_atoms, const char *const *names) {
  pmb_traj *t = pmb_traj_open_xyz(path, n_atoms, names);
  if (t) t->kind = 2;
  return t;
}

int pmb_traj_set_minimal_image(pmb_traj *t, const double *mass, const int *molecule, int n_pairs,
                               const int *pairs, const double box[3], const double origin[3]) {
  if (!t || !mass || !molecule || n_pairs < 0 || (n_pairs > 0 && !pairs) || !box || !origin)
    return set_error("null argument"), PMB_ERR_ARG;
  if (t->kind != 0) return set_error("minimal image applies to DCD trajectories"), PMB_ERR_ARG;
  if (t->started || t->frames) return set_error("minimal image must be set before the first frame"), PMB_ERR_STATE;
  const int n = t->n_atoms;
  for (int c = 0; c < 3; c++)
    if (!(box[c] > 0) || !std::isfinite(origin[c])) return set_error("box edges > 0, finite origin"), PMB_ERR_ARG;
  int nmol = 0;
  for (int i = 0; i < n; i++) {
    if (molecule[i] < 0 || molecule[i] >= n) return set_error("molecule index out of range"), PMB_ERR_ARG;
    nmol = std::max(nmol, molecule[i] + 1);
  }
  MinimalImage *mi = new MinimalImage();
  mi->atoms.resize(nmol);
  mi->pairs.resize(nmol);
  for (int i = 0; i < n; i++) mi->atoms[molecule[i]].push_back(i);
  for (int k = 0; k < n_pairs; k++) {
    int a = pairs[2 * k], b = pairs[2 * k + 1];
    if (a < 0 || a >= n || b < 0 || b >= n || molecule[a] != molecule[b] || a == b) {
      delete mi;
      return set_error("pair " + std::to_string(k) + " does not join two atoms of one molecule"), PMB_ERR_ARG;
    }
    if (a > b) std::swap(a, b);
    mi->pairs[molecule[a]].push_back(std::make_pair(a, b));
  }
  for (auto &p : mi->pairs) std::sort(p.begin(), p.end());
  // molecule ids without atoms leave empty molecules, which the transform skips
  std::vector<std::vector<int>> atoms;
  std::vector<std::vector<std::pair<int, int>>> prs;
  for (int m = 0; m < nmol; m++)
    if (!mi->atoms[m].empty()) {
      atoms.push_back(mi->atoms[m]);
      prs.push_back(mi->pairs[m]);
    }
  mi->atoms.swap(atoms);
  mi->pairs.swap(prs);
  mi->mass.assign(mass, mass + n);
  // PeriodicBoundaryConditions::set (topology/PeriodicBoundaryConditions.cpp:32-77) for the
  // orthogonal box (e1, e2, e3) = diag(box): reciprocal edges and the safe distance
  const double lx = box[0], ly = box[1], lz = box[2];
  mi->L[0] = lx;
  mi->L[1] = ly;
  mi->L[2] = lz;
  mi->Lr[0] = (ly * lz) / (lx * (ly * lz));
  mi->Lr[1] = (lz * lx) / (ly * (lz * lx));
  mi->Lr[2] = (lx * ly) / (lz * (lx * ly));
  for (int c = 0; c < 3; c++) mi->origin[c] = origin[c];
  const double dx = (lx * 0.5) * (lx * 0.5), dy = (ly * 0.5) * (ly * 0.5), dz = (lz * 0.5) * (lz * 0.5);
  mi->D = std::min(dx, std::min(dy, dz));
  delete t->minimal;
  t->minimal = mi;
  return PMB_OK;
}

int pmb_md_write_checkpoint(pmb_md *md, const char *config_path, int id, long long first_step,
                            const char *pos_base, const char *vel_base, const char *const *names) {
  if (!md || !config_path || !*config_path || !pos_base || !vel_base || !names)
    return set_error("null argument"), PMB_ERR_ARG;
  const double *d_pos = nullptr;
  int n = 0, dev = 0, kind = 0;
  cudaStream_t st = nullptr;
  int rc = md_frame_source(md, &d_pos, &n, &st, &dev);
  if (rc) return rc;
  std::vector<std::string> nm(n);
  for (int i = 0; i < n; i++) {
    if (!names[i]) return set_error("null atom name"), PMB_ERR_ARG;
    nm[i] = names[i];
  }
  std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n);
  long long steps = 0;
  rc = pmb_md_get_checkpoint(md, x.data(), v.data(), nullptr, &steps);
  if (rc) return rc;
  unsigned long long seed = 0;
  long long noise_steps = 0;  // the first box's stream: its seed and step count
  md_noise(md, &kind, &seed, &noise_steps);
  const std::string pos_file = std::string(pos_base) + std::to_string(id) + ".pos";
  const std::string vel_file = std::string(vel_base) + std::to_string(id) + ".vel";
  if (!write_file(pos_file, xyz_text(n, nm, x.data())))
    return set_error("cannot write " + pos_file), PMB_ERR_ARG;
  if (!write_file(vel_file, xyz_text(n, nm, v.data())))
    return set_error("cannot write " + vel_file), PMB_ERR_ARG;
  // CheckpointConfigWriter::write (io/CheckpointConfigWriter.cpp:11-25); the leapfrog and
  // Langevin integrators write nothing after #Integrator (Integrator::streamWrite)
  std::ostringstream o;
  o << "!Checkpoint File!" << std::endl
    << "#ID" << std::endl
    << id << std::endl
    << "#Step" << std::endl
    << first_step + steps << std::endl
    << "#Random" << std::endl
    << "philox4x32-10 " << seed << " " << (kind == PMB_LANGEVIN ? 2 * noise_steps : 0) << std::endl
    << "#Integrator" << std::endl
    << std::endl;
  const std::string tmp = std::string(config_path) + ".tmp";
  if (!write_file(tmp, o.str()) || std::rename(tmp.c_str(), config_path) != 0)
    return set_error(std::string("cannot write ") + config_path), PMB_ERR_ARG;
  // the previous checkpoint's files go (OutputCheckpoint::doIt)
  std::remove((std::string(pos_base) + std::to_string(id - 1) + ".pos").c_str());
  std::remove((std::string(vel_base) + std::to_string(id - 1) + ".vel").c_str());
  return PMB_OK;
}

int pmb_traj_flush(pmb_traj *t) {
  if (!t) return set_error("null trajectory"), PMB_ERR_ARG;
  const int rc = t->flush();
  if (rc) set_error(t->err_msg);
  return rc;
}

int pmb_traj_frames(pmb_traj *t, long long *frames) {
  if (!t || !frames) return set_error("null argument"), PMB_ERR_ARG;
  const int rc = t->flush();
  *frames = t->frames;
  return rc;
}

int pmb_traj_close(pmb_traj *t) {
  if (!t) return PMB_OK;
  const int rc = t->flush();
  const std::string msg = t->err_msg;
  delete t;
  if (rc) set_error(msg);
  return rc;
}

}  // extern "C"
