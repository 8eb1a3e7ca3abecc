// adapter_harness.cpp -- drives the C++ drop-in (csrc/cuda_accelerator.h)
// the way libraw_enhanced's pipeline calls a GPUAccelerator: host
// ImageBufferFloat buffers, the post-demosaic stages aliased in == out
// (core/cpu_accelerator.h:137,167 call them with (rgb_buffer, rgb_buffer)).
//
//   adapter_harness <raw.f32> <width> <height> <filters> <out prefix>
//
// raw.f32 is the reference's sparse (H, W, 3) float raw buffer.  Writes
// <prefix>amaze.f32, <prefix>defringe.f32, <prefix>axial.f32 (float32
// (H, W, 3) each) after demosaic_bayer_amaze (cam_mul 2, 1, 1.5, 1;
// maximum 1), defringe (10, 0.1, 0.15, 10, off, 0.3) and
// ca_axial_cleanup (6, 1e-4, 0.3).  Exit 0 on success.
//
// Built with -DLRE_USE_REFERENCE_TYPES against the reference's
// core/accelerator.h, the adapter uses libraw_enhanced::ImageBuffer /
// ImageBufferFloat themselves; without it, the adapter's layout-identical
// structs.
#ifdef LRE_USE_REFERENCE_TYPES
#include "accelerator.h"
#endif
#include "libraw_enhanced_b200/csrc/cuda_accelerator.h"

#include <cstdio>
#include <cstdlib>
#include <vector>

static bool save(const std::vector<float>& v, const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = std::fwrite(v.data(), sizeof(float), v.size(), f) == v.size();
  return std::fclose(f) == 0 && ok;
}

int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s raw.f32 width height filters out_prefix\n", argv[0]);
    return 2;
  }
  const size_t w = std::strtoul(argv[2], nullptr, 10), h = std::strtoul(argv[3], nullptr, 10);
  const uint32_t filters = (uint32_t)std::strtoul(argv[4], nullptr, 0);
  const std::string prefix = argv[5];
  std::vector<float> raw(w * h * 3), rgb(w * h * 3);
  FILE* f = std::fopen(argv[1], "rb");
  if (!f || std::fread(raw.data(), sizeof(float), raw.size(), f) != raw.size()) {
    std::fprintf(stderr, "cannot read %s\n", argv[1]);
    return 2;
  }
  std::fclose(f);

  lre::CudaAccelerator acc;
  if (!acc.initialize(0)) {
    std::fprintf(stderr, "initialize: %s\n", acc.last_error().c_str());
    return 3;
  }
  lre::CudaAccelerator::ImageBufferFloat in, out;
  in.image = reinterpret_cast<float(*)[3]>(raw.data());
  in.width = w;
  in.height = h;
  in.channels = 3;
  out.image = reinterpret_cast<float(*)[3]>(rgb.data());
  out.width = w;
  out.height = h;
  out.channels = 3;
  const float cam_mul[4] = {2.0f, 1.0f, 1.5f, 1.0f};
  if (!acc.demosaic_bayer_amaze(in, out, filters, cam_mul, 1.0f)) {
    std::fprintf(stderr, "demosaic_bayer_amaze: %s\n", acc.last_error().c_str());
    return 4;
  }
  if (!save(rgb, prefix + "amaze.f32")) return 5;
  if (!acc.defringe(out, out, 10.0f, 0.1f, 0.15f, 10.0f, false, 0.3f)) {
    std::fprintf(stderr, "defringe: %s\n", acc.last_error().c_str());
    return 4;
  }
  if (!save(rgb, prefix + "defringe.f32")) return 5;
  if (!acc.ca_axial_cleanup(out, out, 6, 1e-4f, 0.3f)) {
    std::fprintf(stderr, "ca_axial_cleanup: %s\n", acc.last_error().c_str());
    return 4;
  }
  if (!save(rgb, prefix + "axial.f32")) return 5;
  // the reference's default arguments compile: gamma_correct(in, out)
  std::vector<float> g(rgb.size());
  lre::CudaAccelerator::ImageBufferFloat gb = out;
  gb.image = reinterpret_cast<float(*)[3]>(g.data());
  if (!acc.gamma_correct(out, gb)) {
    std::fprintf(stderr, "gamma_correct: %s\n", acc.last_error().c_str());
    return 4;
  }
  if (!save(g, prefix + "gamma.f32")) return 5;
  return 0;
}
