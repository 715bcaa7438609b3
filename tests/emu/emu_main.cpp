// emu_main.cpp -- TEST INFRASTRUCTURE: drives the library's public C API in
// the CPU emulation build.
//   emu_main <op> ix iy iz kx ky kz <param> image.raw psf.raw out.raw
// op: convolve | rl | blind | jvc | sjvc | wiener (param = iterations or epsilon).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/clarity.h"
#include "../../include/clarity_ext.h"

static std::vector<float> read_raw(const char* path, size_t n) {
  std::vector<float> v(n);
  FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), sizeof(float), n, f) != n) {
    std::fprintf(stderr, "cannot read %s\n", path);
    std::exit(2);
  }
  std::fclose(f);
  return v;
}

int main(int argc, char** argv) {
  if (argc != 12) {
    std::fprintf(stderr, "usage: emu_main op ix iy iz kx ky kz param img psf out\n");
    return 2;
  }
  const std::string op = argv[1];
  Clarity_Dim3 id{std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4])};
  Clarity_Dim3 kd{std::atoi(argv[5]), std::atoi(argv[6]), std::atoi(argv[7])};
  const double param = std::atof(argv[8]);
  const size_t ni = (size_t)id.x * id.y * id.z, nk = (size_t)kd.x * kd.y * kd.z;
  std::vector<float> img = read_raw(argv[9], ni), psf = read_raw(argv[10], nk), out(ni);
  if (Clarity_Register() != CLARITY_SUCCESS) return 3;
  ClarityResult_t r;
  if (op == "convolve")
    r = Clarity_Convolve(img.data(), id, psf.data(), kd, out.data());
  else if (op == "rl")
    r = Clarity_MaximumLikelihoodDeconvolve(img.data(), id, psf.data(), kd, out.data(), (int)param);
  else if (op == "blind")
    r = Clarity_BlindMaximumLikelihoodDeconvolve(img.data(), id, psf.data(), kd, out.data(),
                                                 (int)param);
  else if (op == "jvc")
    r = Clarity_JansenVanCittertDeconvolve(img.data(), id, psf.data(), kd, out.data(), (int)param);
  else if (op == "sjvc") {  // smoothed JVC: interval 2, sigma (1.0, 1.5, 0.7)
    float sx = 1.0f, sy = 1.5f, sz = 0.7f;
    float* sig[3] = {&sx, &sy, &sz};
    r = Clarity_SmoothedJansenVanCittertDeconvolve(img.data(), id, psf.data(), kd, out.data(),
                                                   (unsigned)param, 2u, sig);
  } else if (op == "convolve_noalloc")  // emulated device memory is host memory
    r = clarityx_convolve_noalloc(img.data(), id, psf.data(), kd, out.data(), nullptr);
  else if (op == "wiener")
    r = Clarity_WienerDeconvolve(img.data(), id, psf.data(), kd, out.data(), (float)param);
  else
    return 2;
  if (r != CLARITY_SUCCESS) {
    std::fprintf(stderr, "%s returned %d\n", op.c_str(), (int)r);
    return 4;
  }
  Clarity_UnRegister();
  FILE* f = std::fopen(argv[11], "wb");
  std::fwrite(out.data(), sizeof(float), ni, f);
  std::fclose(f);
  return 0;
}
