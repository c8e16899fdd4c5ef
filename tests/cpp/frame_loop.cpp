// C++ host driving the C ABI through kf_gfusion.hpp, the way the reference's main loop
// drives gFusion (src/kinect.cpp:654-695): reads uint16 depth frames from a file, runs the
// frame step, prints one line per frame: tracked flag and the 16 pose values.
//   frame_loop <frames.u16> <n_frames> <volume size> <dim m> <mu m> <x y z of pose 0...16 values>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "kf_gfusion.hpp"

int main(int argc, char** argv) {
  if (argc < 6 + 16) {
    std::fprintf(stderr, "usage: frame_loop frames.u16 n size dim mu pose0[16 column-major]\n");
    return 2;
  }
  const char* path = argv[1];
  const int n = std::atoi(argv[2]);
  kf_config cfg = kf::default_config();
  cfg.nx = cfg.ny = cfg.nz = std::atoi(argv[3]);
  cfg.dim_x = cfg.dim_y = cfg.dim_z = (float)std::atof(argv[4]);
  cfg.mu = (float)std::atof(argv[5]);
  cfg.iterations[0] = 10;
  cfg.iterations[1] = 5;
  cfg.iterations[2] = 4;
  cfg.quirks = KF_QUIRKS_TRACKING;
  kf::Pose pose0;
  for (int i = 0; i < 16; ++i) pose0[i] = std::atof(argv[6 + i]);
  const kf_intrinsics intr = {365.0f, 365.0f, 256.0f, 212.0f, 512, 424};
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return 3;
  std::vector<uint16_t> frame(512 * 424);
  try {
    kf::GFusion fusion(cfg, intr);
    fusion.Reset(pose0, false);
    for (int k = 0; k < n; ++k) {
      if (std::fread(frame.data(), 2, frame.size(), f) != frame.size()) return 4;
      const bool tracked = fusion.frameStep(frame.data());
      const kf::Pose p = fusion.getPose();
      std::printf("%d", tracked ? 1 : 0);
      for (double v : p) std::printf(" %.17g", v);
      std::printf("\n");
    }
    kf::MCubes mc(fusion);
    mc.setIsolevel(0.0f);
    mc.generateMarchingCubes();
    std::printf("triangles %d\n", mc.getNumberTriangles() / 3);
  } catch (const kf::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 5;
  }
  std::fclose(f);
  return 0;
}
