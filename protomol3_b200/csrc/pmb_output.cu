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
//
// pmb_md_write_frame takes a frame off the device without stopping it: a device-to-device
// snapshot of the positions on the system's stream (the next step waits only for that), the
// snapshot's copy into one of three pinned host buffers on the trajectory's own stream, and a
// writer thread per trajectory that waits for the copy and appends the frame.  The caller waits
// only when all three buffers are still in flight.
#include <cuda_runtime.h>

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

}  // namespace

struct pmb_traj {
  int kind = 0;  // 0 DCD, 1 XYZ
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
    std::ostringstream o;
    o << n_atoms << std::endl;
    o.precision(15);
    for (int i = 0; i < n_atoms; i++) {
      o << names[i] << "\t";
      for (int c = 0; c < 3; c++) {
        o.width(24);
        o << pos[3 * i + c];
      }
      o << std::endl;
    }
    std::FILE *x = std::fopen(path.c_str(), "wb");
    if (!x) return PMB_ERR_ARG;
    const std::string s = o.str();
    const bool ok = std::fwrite(s.data(), 1, s.size(), x) == s.size();
    std::fclose(x);
    frames++;
    return ok ? PMB_OK : PMB_ERR_ARG;
  }

  int write(const double *pos) { return kind == 0 ? write_dcd(pos) : write_xyz(pos); }

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

int pmb_md_write_frame(pmb_md *md, pmb_traj *t) {
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
  if (cudaMemcpyAsync(sg.dev, d_pos, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      cudaEventRecord(sg.taken, st) != cudaSuccess || cudaStreamWaitEvent(t->copy, sg.taken, 0) != cudaSuccess ||
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
