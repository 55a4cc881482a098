// Test-infrastructure harness: ProtoMol 3's own trajectory writers, compiled from the reference
// sources by oracle/Makefile, writing given frames, so tests can compare the files the
// library's writers produce with the reference's byte for byte.
//   DCDTrajectoryWriter as OutputDCDTrajectory::doInitialize makes it (output/OutputDCDTrajectory.cpp:
//   27-43: timestep argument 1.0, first step from the configuration, native byte order), one
//   write() per frame (io/DCDTrajectoryWriter.cpp)
//   XYZWriter::write(coords, names) (io/XYZWriter.cpp), as OutputFinalXYZPos uses it
//   XYZTrajectoryWriter opened and written as OutputXYZTrajectoryForce does
//   (output/OutputXYZTrajectoryForce.cpp:30-44), one write() per frame
//   CheckpointConfigWriter::write (io/CheckpointConfigWriter.cpp:11-25) with the reference's
//   Random and a LeapfrogIntegrator, as OutputCheckpoint::WriteConfig calls it
#include <protomol/base/Report.h>
using namespace ProtoMol::Report;

#include <protomol/base/Random.h>
#include <protomol/force/ForceGroup.h>
#include <protomol/integrator/leapfrog/LeapfrogIntegrator.h>
#include <protomol/io/CheckpointConfigWriter.h>
#include <protomol/io/DCDTrajectoryWriter.h>
#include <protomol/io/XYZTrajectoryWriter.h>
#include <protomol/io/XYZWriter.h>
#include <protomol/type/Vector3DBlock.h>

#include <string>
#include <vector>

using namespace ProtoMol;

static void fill(Vector3DBlock &v, const double *p, int n) {
  v.resize(n);
  for (int i = 0; i < n; i++)
    for (int c = 0; c < 3; c++) v[i][c] = p[3 * i + c];
}

extern "C" int ref_write_dcd(const char *path, int n_atoms, int n_frames, const double *frames,
                             double timestep, int first_step) {
  DCDTrajectoryWriter w(std::string(path), timestep, (unsigned int)first_step);
  if (!w.open()) return 1;
  Vector3DBlock v;
  for (int f = 0; f < n_frames; f++) {
    fill(v, frames + 3 * (size_t)n_atoms * f, n_atoms);
    if (!w.write(v)) return 2;
  }
  w.close();
  return 0;
}

extern "C" int ref_write_xyz(const char *path, int n_atoms, const double *pos, const char *const *names) {
  const std::string fn(path);
  XYZWriter w(fn);
  Vector3DBlock v;
  fill(v, pos, n_atoms);
  std::vector<std::string> nm(names, names + n_atoms);
  return w.write(v, nm) ? 0 : 1;
}

extern "C" int ref_write_xyz_trajectory(const char *path, int n_atoms, int n_frames, const double *frames,
                                        const char *const *names) {
  XYZTrajectoryWriter w((std::string(path)));
  if (!w.open()) return 1;
  std::vector<std::string> nm(names, names + n_atoms);
  Vector3DBlock v;
  for (int f = 0; f < n_frames; f++) {
    fill(v, frames + 3 * (size_t)n_atoms * f, n_atoms);
    if (!w.write(v, nm)) return 2;
  }
  w.close();
  return 0;
}

extern "C" int ref_write_checkpoint_config(const char *path, int id, int step) {
  CheckpointConfigWriter w;
  if (!w.open(std::string(path))) return 1;
  LeapfrogIntegrator integ(1.0, new ForceGroup());
  if (!w.write(id, step, Random::Instance(), &integ)) return 2;
  w.close();
  return 0;
}
