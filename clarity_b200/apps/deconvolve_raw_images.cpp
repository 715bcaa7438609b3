// deconvolve_raw_images -- the reference's example application
// (apps/DeconvolveRawImages/DeconvolveRawImages.cxx) on this library: reads
// uint16 raw image and PSF volumes, runs 5 Richardson-Lucy iterations and
// writes the uint16 result.  Same command line; the uint16 <-> float casts run
// on the GPU (clarityx_ml_u16), so only uint16 data crosses the bus.
//
//   deconvolve_raw_images <image> <x> <y> <z> <psf> <x> <y> <z> <output>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "clarity.h"
#include "clarity_ext.h"

static bool read_u16(const char* path, std::vector<uint16_t>* v) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  const size_t got = std::fread(v->data(), sizeof(uint16_t), v->size(), f);
  std::fclose(f);
  return got == v->size();
}

int main(int argc, char** argv) {
  if (argc < 10) {
    std::printf("Usage: %s <image filename> <x> <y> <z> <psf filename> <x> <y> <z> "
                "<output file name>\n", argv[0]);
    return 1;
  }
  const Clarity_Dim3 id{std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4])};
  const Clarity_Dim3 kd{std::atoi(argv[6]), std::atoi(argv[7]), std::atoi(argv[8])};
  if (id.x <= 0 || id.y <= 0 || id.z <= 0 || kd.x <= 0 || kd.y <= 0 || kd.z <= 0) {
    std::printf("ERROR: dimensions must be positive\n");
    return 1;
  }
  std::vector<uint16_t> img((size_t)id.x * id.y * id.z), psf((size_t)kd.x * kd.y * kd.z);
  std::vector<uint16_t> out(img.size());
  if (!read_u16(argv[1], &img)) {
    std::printf("Error reading input image file\n");
    return 1;
  }
  if (!read_u16(argv[5], &psf)) {
    std::printf("Error reading PSF file\n");
    return 1;
  }
  ClarityResult_t r = Clarity_Register();
  if (r == CLARITY_SUCCESS) r = clarityx_ml_u16(img.data(), id, psf.data(), kd, out.data(), 5);
  if (r != CLARITY_SUCCESS) {
    std::printf("ERROR: %s (%s)\n", Clarity_ResultString(r), clarityx_last_error());
    return 2;
  }
  Clarity_UnRegister();
  FILE* f = std::fopen(argv[9], "wb");
  if (!f || std::fwrite(out.data(), sizeof(uint16_t), out.size(), f) != out.size()) {
    std::printf("ERROR: Could not write file '%s'\n", argv[9]);
    if (f) std::fclose(f);
    return 1;
  }
  std::fclose(f);
  std::printf("Input image file name: %s\n", argv[1]);
  std::printf("Input image dimensions: %d x %d x %d\n", id.x, id.y, id.z);
  std::printf("Input point-spread function file name: %s\n", argv[5]);
  std::printf("Input point-spread function dimensions: %d x %d x %d\n", kd.x, kd.y, kd.z);
  std::printf("Output file name: %s\n", argv[9]);
  return 0;
}
