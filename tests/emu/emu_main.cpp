// emu_main.cpp -- TEST INFRASTRUCTURE: drives the library's public C API in
// the CPU emulation build.
//   emu_main <op> ix iy iz kx ky kz <param> image.raw psf.raw out.raw
// op: convolve | rl | blind | jvc | sjvc | wiener (param = iterations or epsilon).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>

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

// Learned-start convolution kernels on deterministic BF16 data: dims (W, H,
// D) = id, channels (c1, c2, cout) = kd.  Writes the inputs and results as
// float32 files prefix.{x1,x2,w,b,dy,y,dx,dw,db} for the test to check.
static float hval(uint32_t i, float scale) {
  const uint32_t h = i * 2654435761u + 12345u;
  return scale * ((float)((h >> 8) % 2001) / 1000.0f - 1.0f);
}
static void dump(const std::string& path, const std::vector<float>& v) {
  FILE* f = std::fopen(path.c_str(), "wb");
  std::fwrite(v.data(), sizeof(float), v.size(), f);
  std::fclose(f);
}
static int nn_conv_case(Clarity_Dim3 id, Clarity_Dim3 kd, int relu, const char* prefix) {
  const int W = id.x, H = id.y, D = id.z, c1 = kd.x, c2 = kd.y, co = kd.z, cin = c1 + c2;
  const size_t V = (size_t)D * H * W, V2 = c2 ? V / 8 : 0;
  auto mk = [](size_t n, uint32_t seed, float scale, std::vector<__nv_bfloat16>* b,
               std::vector<float>* f) {
    b->resize(n);
    f->resize(n);
    for (size_t i = 0; i < n; ++i) {
      (*b)[i] = __float2bfloat16_rn(hval((uint32_t)i * 7u + seed, scale));
      (*f)[i] = __bfloat162float((*b)[i]);
    }
  };
  std::vector<__nv_bfloat16> x1, x2, wq, dy, y(V * co), dx(V * cin);
  std::vector<float> fx1, fx2, fw, fdy, fb(co);
  mk(V * c1, 1, 1.0f, &x1, &fx1);
  mk(V2 * c2, 2, 1.0f, &x2, &fx2);
  mk((size_t)co * 27 * cin, 3, 0.1f, &wq, &fw);
  mk(V * co, 4, 1.0f, &dy, &fdy);
  for (int i = 0; i < co; ++i) fb[i] = hval(100 + i, 0.2f);
  ClarityResult_t r = clarityx_nn_conv3(x1.data(), c1, c2 ? x2.data() : nullptr, c2, D, H, W,
                                        wq.data(), fb.data(), co, relu, nullptr, y.data(), nullptr);
  if (r != CLARITY_SUCCESS) return 4;
  std::vector<float> dw((size_t)co * 27 * cin, 0.f), db(co, 0.f);
  r = clarityx_nn_conv3_wgrad(x1.data(), c1, c2 ? x2.data() : nullptr, c2, D, H, W, dy.data(), co,
                              dw.data(), db.data(), nullptr);
  if (r != CLARITY_SUCCESS) return 4;
  std::vector<float> fy(y.size());
  for (size_t i = 0; i < y.size(); ++i) fy[i] = __bfloat162float(y[i]);
  const std::string p = prefix;
  dump(p + ".x1", fx1);
  dump(p + ".x2", fx2);
  dump(p + ".w", fw);
  dump(p + ".b", fb);
  dump(p + ".dy", fdy);
  dump(p + ".y", fy);
  dump(p + ".dw", dw);
  dump(p + ".db", db);
  return 0;
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
  if (op == "nnconv") return nn_conv_case(id, kd, (int)param, argv[11]);
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
  } else if (op == "correlate") {  // emulated device memory is host memory
    r = clarityx_correlate_device(img.data(), id, psf.data(), kd, out.data(), nullptr);
  } else if (op == "rlcorr") {
    r = clarityx_ml_correlate_device(img.data(), id, psf.data(), kd, out.data(), (int)param,
                                     nullptr);
  } else if (op == "accel") {  // accelerated RL, emulated device memory is host memory
    r = clarityx_ml_accel_device(img.data(), id, psf.data(), kd, nullptr, out.data(), (int)param,
                                 nullptr, nullptr);
  } else if (op == "blindpsf") {  // blind ML with 3 PSF steps per iteration; out = object
    std::vector<float> pout(nk);
    r = clarityx_blind_ml_psf_device(img.data(), id, psf.data(), kd, out.data(), pout.data(),
                                     (int)param, 3, nullptr);
  } else if (op == "batch" || op == "batchp") {
    // three volumes of different sizes in one batched call (emulated device
    // memory is host memory); each must equal its single-volume solve.
    // batchp: the persistent launch, whose iterations use the runtime-planned
    // kernels: equal bit for bit when the single solves do too (CLARITY_STATIC
    // = 0; the host compiler contracts no multiply-add here), else within
    // 2e-6 relative L2
    const int n = 3;
    Clarity_Dim3 bid[n] = {id, {id.x / 2 > 0 ? id.x / 2 : 1, id.y, id.z}, id};
    {
      int info[16];
      const Clarity_Dim3 w1{bid[1].x + kd.x, bid[1].y + kd.y, bid[1].z + kd.z};
      if (clarityx_plan_info(w1, info, 16) != CLARITY_SUCCESS) bid[1] = id;  // unsupported box
    }
    std::vector<float> vin[n], vout[n];
    const float* ip[n];
    const float* kp[n];
    float* op_[n];
    Clarity_Dim3 bkd[n] = {kd, kd, kd};
    for (int v = 0; v < n; ++v) {
      vin[v].resize((size_t)bid[v].x * bid[v].y * bid[v].z);
      for (int z = 0; z < bid[v].z; ++z)
        for (int y = 0; y < bid[v].y; ++y)
          for (int x = 0; x < bid[v].x; ++x)
            vin[v][((size_t)z * bid[v].y + y) * bid[v].x + x] =
                img[((size_t)z * id.y + y) * id.x + x] * (1.0f + 0.25f * v);
      vout[v].assign(vin[v].size(), -1.f);
      ip[v] = vin[v].data();
      kp[v] = psf.data();
      op_[v] = vout[v].data();
    }
    const bool pers = op == "batchp";
    const char* sm = std::getenv("CLARITY_STATIC");
    const bool exact = !pers || (sm && std::atoi(sm) == 0);
    r = clarityx_ml_batch_device(n, ip, bid, kp, bkd, op_, (int)param,
                                 pers ? CLARITYX_BATCH_PERSISTENT : CLARITYX_BATCH_GRAPH,
                                 nullptr);
    for (int v = 0; v < n && r == CLARITY_SUCCESS; ++v) {
      std::vector<float> one(vin[v].size());
      r = Clarity_MaximumLikelihoodDeconvolve(vin[v].data(), bid[v], psf.data(), kd, one.data(),
                                              (int)param);
      if (r != CLARITY_SUCCESS) break;
      double num = 0, den = 0;
      for (size_t i = 0; i < one.size(); ++i) {
        const double d = (double)one[i] - vout[v][i];
        num += d * d;
        den += (double)one[i] * one[i];
      }
      const bool same = std::memcmp(one.data(), vout[v].data(), 4 * one.size()) == 0;
      if (exact ? !same : !(num <= 4e-12 * den)) {
        std::fprintf(stderr, "batch volume %d differs from its single solve (rel-L2 %.3g)\n", v,
                     den > 0 ? std::sqrt(num / den) : 0.0);
        return 5;
      }
    }
    out = vout[0];
  } else if (op == "convolve_noalloc")  // emulated device memory is host memory
    r = clarityx_convolve_noalloc(img.data(), id, psf.data(), kd, out.data(), nullptr);
  else if (op == "wiener")
    r = Clarity_WienerDeconvolve(img.data(), id, psf.data(), kd, out.data(), (float)param);
  else if (op == "idiv" || op == "idiva")  // I-divergence restoration, alpha 0 or 1e-4
    r = clarityx_idiv_deconvolve_device(img.data(), id, psf.data(), kd, out.data(), (int)param,
                                        op == "idiva" ? 1e-4f : 0.f, nullptr);
  else if (op == "u16") {  // raw uint16 volumes (inputs hold integers); out = the uint16 result
    std::vector<uint16_t> gi(ni), gk(nk), go(ni);
    for (size_t i = 0; i < ni; ++i) gi[i] = (uint16_t)img[i];
    for (size_t i = 0; i < nk; ++i) gk[i] = (uint16_t)psf[i];
    r = clarityx_ml_u16(gi.data(), id, gk.data(), kd, go.data(), (int)param);
    for (size_t i = 0; i < ni; ++i) out[i] = (float)go[i];
  } else
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
