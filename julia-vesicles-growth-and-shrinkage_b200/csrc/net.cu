// C ABI of the learned psi-preconditioner network (declared in include/vsav.h):
// parameters, GPU forward / gradient / Adam training on crop sets, and the
// fused tensor-core inference kernel on plain input batches.
#include "../../include/vsav.h"
#include "net.cuh"
#include "net_apply.cuh"
#include "net_tc.cuh"

#include <string>

using namespace vsav;

struct vsav_net {
  Net n;
  int device = 0;
  std::string err;
  uint32_t* frag = nullptr;        // packed mma fragments of the BF16 weights
  float* fbias = nullptr;
  uint4* timg = nullptr;           // B operands of the tcgen05 kernel (net_pack_tc image)
  int* derr = nullptr;             // error word of the tcgen05 kernel's bounded waits
  float* tbuf = nullptr;           // gathered targets of a training batch
  bool frags_dirty = true;
};

namespace {

thread_local std::string g_net_create_error;

template <typename F>
int nguard(vsav_net* h, F&& f) {
  if (!h) return VSAV_E_INVALID;
  try {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e));
    return f();
  } catch (const std::exception& e) {
    h->err = e.what();
    return (h->err.rfind("CUDA", 0) == 0) ? VSAV_E_CUDA : VSAV_E_INVALID;
  }
}

void refresh_frags(vsav_net* h) {
  if (!h->frags_dirty) return;
  std::vector<float> wb(NET_NPARAM);
  VSAV_CUDA(cudaMemcpyAsync(wb.data(), h->n.wb, NET_NPARAM * 4, cudaMemcpyDeviceToHost, h->n.st));
  VSAV_CUDA(cudaStreamSynchronize(h->n.st));
  std::vector<uint32_t> fr(NF_WORDS);
  std::vector<float> bias(NF_BIAS, 0.f);
  net_pack(wb.data(), fr.data(), bias.data());
  std::vector<uint16_t> img(NT_WBYTES / 2);
  net_pack_tc(wb.data(), img.data());
  VSAV_CUDA(cudaMemcpyAsync(h->frag, fr.data(), NF_WORDS * 4, cudaMemcpyHostToDevice, h->n.st));
  VSAV_CUDA(cudaMemcpyAsync(h->fbias, bias.data(), NF_BIAS * 4, cudaMemcpyHostToDevice, h->n.st));
  VSAV_CUDA(cudaMemcpyAsync(h->timg, img.data(), NT_WBYTES, cudaMemcpyHostToDevice, h->n.st));
  VSAV_CUDA(cudaStreamSynchronize(h->n.st));
  h->frags_dirty = false;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// weighted loss sums of the current network on crops [c0, c0 + B) of a set
void batch_loss(vsav_net* h, const float* x, const float* t, const float* w, long long c0, int B, int S, int kind,
                float op_c0, double* se, double* st2) {
  Net& n = h->n;
  const long long per_in = 2LL * S * S, per_out = (long long)(S - 10) * (S - 10);
  VSAV_CUDA(cudaMemcpyAsync(n.act[0], x + c0 * per_in, (size_t)B * per_in * 4, cudaMemcpyDefault, n.st));
  n.forward<false>(B, S, S);
  if (kind == 1) n.loss_res(t + c0 * per_out, B, S, op_c0, n.g0, n.g1, w ? w + c0 : nullptr);
  else n.loss(t + c0 * per_out, (long long)B * per_out, 1, n.g0, w ? w + c0 : nullptr, per_out);
  double ls[2];
  VSAV_CUDA(cudaMemcpyAsync(ls, n.lsum, 16, cudaMemcpyDeviceToHost, n.st));
  VSAV_CUDA(cudaStreamSynchronize(n.st));
  *se += ls[0];
  *st2 += ls[1];
}

}  // namespace

extern "C" {

int vsav_net_nparams(void) { return NET_NPARAM; }
const char* vsav_net_last_error(const vsav_net* h) { return h ? h->err.c_str() : g_net_create_error.c_str(); }

int vsav_net_create(int64_t cap_pixels, int32_t device, vsav_net** out) {
  if (!out || cap_pixels <= 0) return VSAV_E_INVALID;
  *out = nullptr;
  auto* h = new vsav_net();
  h->device = device;
  try {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e));
    h->n.init(cap_pixels, (int)std::min<long long>(cap_pixels / 121, 1 << 20));
    h->frag = h->n.alloc<uint32_t>(NF_WORDS);
    h->fbias = h->n.alloc<float>(NF_BIAS);
    h->timg = h->n.alloc<uint4>(NT_WBYTES / 16);
    h->derr = h->n.alloc<int>(1);
    h->tbuf = h->n.alloc<float>((size_t)cap_pixels);
  } catch (const std::exception& ex) {
    g_net_create_error = ex.what();
    delete h;
    return g_net_create_error.rfind("CUDA", 0) == 0 ? VSAV_E_CUDA : VSAV_E_INVALID;
  }
  *out = h;
  return VSAV_OK;
}

int vsav_net_destroy(vsav_net* h) {
  if (!h) return VSAV_E_INVALID;
  cudaSetDevice(h->device);
  delete h;
  return VSAV_OK;
}

int vsav_net_set_params(vsav_net* h, const double* theta) {
  return nguard(h, [&] {
    if (!theta) throw std::runtime_error("theta is NULL");
    h->n.set_params(theta);
    h->frags_dirty = true;
    return VSAV_OK;
  });
}

int vsav_net_get_params(vsav_net* h, double* theta, int32_t rounded) {
  return nguard(h, [&] {
    if (!theta) throw std::runtime_error("theta is NULL");
    h->n.get_params(theta, rounded);
    return VSAV_OK;
  });
}

int vsav_net_forward(vsav_net* h, const float* x, int32_t B, int32_t H, int32_t W, int32_t periodic, int32_t impl,
                     float* out) {
  return nguard(h, [&] {
    Net& n = h->n;
    const bool P = periodic != 0;
    n.check(B, H, W, P);
    const int Ho = P ? H : H - 10, Wo = P ? W : W - 10;
    if (impl == 1 || impl == 2) {
      if (!P) throw std::runtime_error("the fused kernel is periodic only");
      if (H % NA_T || W % NA_T || (H & (H - 1)) || (W & (W - 1)))
        throw std::runtime_error("the fused kernel needs H and W powers of two, multiples of 32");
      refresh_frags(h);
      VSAV_CUDA(cudaMemcpyAsync(n.act[0], x, (size_t)B * 2 * H * W * 4, cudaMemcpyDefault, n.st));
      if (impl == 1) {
        VSAV_CUDA(cudaFuncSetAttribute(k_net_apply<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, NA_SMEM));
        dim3 grid((H / NA_T) * (W / NA_T), B);
        k_net_apply<0><<<grid, NA_THREADS, NA_SMEM, n.st>>>(n.act[0], nullptr, nullptr, n.act[NET_NL], H, W, 1, h->frag,
                                                            h->fbias); VSAV_COUNT_LAUNCH();
        VSAV_LAUNCH_CHECK();
      } else {
        VSAV_CUDA(net_tc_attributes<0>());
        int nsm = 0;
        VSAV_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
        const long long tiles = (long long)B * (H / NT_T) * (W / NT_T);
        VSAV_CUDA(cudaMemsetAsync(h->derr, 0, sizeof(int), n.st));
        k_net_apply_tc<0><<<(unsigned)std::min<long long>(tiles, nsm), NT_THREADS, NT_SMEM, n.st>>>(
            n.act[0], nullptr, nullptr, n.act[NET_NL], H, W, 1, B, h->timg, h->fbias, h->derr); VSAV_COUNT_LAUNCH();
        VSAV_LAUNCH_CHECK();
        int e = 0;
        VSAV_CUDA(cudaMemcpyAsync(&e, h->derr, sizeof(int), cudaMemcpyDeviceToHost, n.st));
        VSAV_CUDA(cudaStreamSynchronize(n.st));
        if (e) throw std::runtime_error("CUDA: device-side bound exceeded in the tcgen05 network kernel");
      }
    } else if (impl == 0) {
      VSAV_CUDA(cudaMemcpyAsync(n.act[0], x, (size_t)B * 2 * H * W * 4, cudaMemcpyDefault, n.st));
      if (P) n.forward<true>(B, H, W); else n.forward<false>(B, H, W);
    } else {
      throw std::runtime_error("impl must be 0 (FP32 per layer), 1 (fused, mma.sync) or 2 (fused, tcgen05)");
    }
    VSAV_CUDA(cudaMemcpyAsync(out, n.act[NET_NL], (size_t)B * Ho * Wo * 4, cudaMemcpyDefault, n.st));
    VSAV_CUDA(cudaStreamSynchronize(n.st));
    return VSAV_OK;
  });
}

int vsav_net_grad(vsav_net* h, const float* x, const float* t, int32_t B, int32_t H, int32_t W, int32_t periodic,
                  int32_t loss_kind, double op_c0, double* loss, double* grad) {
  return nguard(h, [&] {
    Net& n = h->n;
    const bool P = periodic != 0;
    n.check(B, H, W, P);
    const int Ho = P ? H : H - 10, Wo = P ? W : W - 10;
    const long long no = (long long)B * Ho * Wo;
    VSAV_CUDA(cudaMemcpyAsync(n.act[0], x, (size_t)B * 2 * H * W * 4, cudaMemcpyDefault, n.st));
    VSAV_CUDA(cudaMemcpyAsync(h->tbuf, t, (size_t)no * 4, cudaMemcpyDefault, n.st));
    if (loss_kind == 1 && (P || H != W)) throw std::runtime_error("the residual loss takes square valid crops");
    if (P) n.forward<true>(B, H, W); else n.forward<false>(B, H, W);
    if (loss_kind == 1) n.loss_res(h->tbuf, B, H, (float)op_c0, n.g0, n.g1);
    else n.loss(h->tbuf, no, 0, n.g1);
    // g1 holds the output gradient; backward uses g0/g1 as ping-pong, so move it
    float* gout = h->tbuf;
    VSAV_CUDA(cudaMemcpyAsync(gout, n.g1, (size_t)no * 4, cudaMemcpyDeviceToDevice, n.st));
    if (P) n.backward<true>(gout, B, H, W); else n.backward<false>(gout, B, H, W);
    double ls[2];
    std::vector<float> g(NET_NPARAM);
    VSAV_CUDA(cudaMemcpyAsync(ls, n.lsum, 16, cudaMemcpyDeviceToHost, n.st));
    VSAV_CUDA(cudaMemcpyAsync(g.data(), n.grad, NET_NPARAM * 4, cudaMemcpyDeviceToHost, n.st));
    VSAV_CUDA(cudaStreamSynchronize(n.st));
    if (loss) *loss = loss_kind == 1 ? ls[0] / std::max(ls[1], 1e-300) : 0.5 * ls[0];
    if (grad)
      for (int k = 0; k < NET_NPARAM; ++k) grad[k] = g[k];
    return VSAV_OK;
  });
}

int vsav_net_train(vsav_net* h, const float* x, const float* t, const float* w, int64_t ncrops, int32_t S,
                   int32_t batch, int32_t nsteps, double lr, uint64_t seed, int32_t flip, int32_t loss_kind,
                   double op_c0, double* losses) {
  return nguard(h, [&] {
    Net& n = h->n;
    if (!x || !t || ncrops <= 0 || batch <= 0 || nsteps < 0) throw std::runtime_error("bad training arguments");
    n.check(batch, S, S, false);
    if (batch > n.cap_batch) throw std::runtime_error("batch too large");
    const long long per_in = 2LL * S * S, per_out = (long long)(S - 10) * (S - 10);
    std::vector<int> idx(batch);
    std::vector<float> sg(batch, 1.f);
    std::vector<double> ls(2 * (size_t)std::max(nsteps, 1));
    double* dls = nullptr;
    VSAV_CUDA(cudaMalloc(&dls, ls.size() * sizeof(double)));
    uint64_t s = seed;
    try {
      for (int it = 0; it < nsteps; ++it) {
        for (int b = 0; b < batch; ++b) {
          idx[b] = (int)(splitmix(s) % (uint64_t)ncrops);
          if (flip) sg[b] = (splitmix(s) & 1) ? -1.f : 1.f;
        }
        VSAV_CUDA(cudaMemcpyAsync(n.idx, idx.data(), batch * sizeof(int), cudaMemcpyHostToDevice, n.st));
        VSAV_CUDA(cudaMemcpyAsync(n.sgn, sg.data(), batch * sizeof(float), cudaMemcpyHostToDevice, n.st));
        const float* sgn = flip ? n.sgn : nullptr;
        k_gather_crops<<<592, 256, 0, n.st>>>(x, n.idx, sgn, batch, per_in, (long long)S * S, n.act[0]); VSAV_COUNT_LAUNCH();
        k_gather_crops<<<592, 256, 0, n.st>>>(t, n.idx, sgn, batch, per_out, per_out, h->tbuf); VSAV_COUNT_LAUNCH();
        if (w) { k_gather_vals<<<(batch + 255) / 256, 256, 0, n.st>>>(w, n.idx, batch, n.wb_batch); VSAV_COUNT_LAUNCH(); }
        VSAV_LAUNCH_CHECK();
        n.forward<false>(batch, S, S);
        if (loss_kind == 1) n.loss_res(h->tbuf, batch, S, (float)op_c0, n.g0, n.g1, w ? n.wb_batch : nullptr);
        else n.loss(h->tbuf, (long long)batch * per_out, 1, n.g1, w ? n.wb_batch : nullptr, per_out);
        VSAV_CUDA(cudaMemcpyAsync(dls + 2 * it, n.lsum, 16, cudaMemcpyDeviceToDevice, n.st));
        VSAV_CUDA(cudaMemcpyAsync(h->tbuf, n.g1, (size_t)batch * per_out * 4, cudaMemcpyDeviceToDevice, n.st));
        n.backward<false>(h->tbuf, batch, S, S);
        n.adam((float)lr);
        // the host index buffer is rewritten next iteration: keep the copy ordered
        VSAV_CUDA(cudaStreamSynchronize(n.st));
      }
      VSAV_CUDA(cudaMemcpyAsync(ls.data(), dls, ls.size() * sizeof(double), cudaMemcpyDeviceToHost, n.st));
      VSAV_CUDA(cudaStreamSynchronize(n.st));
    } catch (...) {
      cudaFree(dls);
      throw;
    }
    cudaFree(dls);
    h->frags_dirty = true;
    if (losses)
      for (int it = 0; it < nsteps; ++it) losses[it] = ls[2 * it] / std::max(ls[2 * it + 1], 1e-300);
    return VSAV_OK;
  });
}

int vsav_net_eval(vsav_net* h, const float* x, const float* t, const float* w, int64_t ncrops, int32_t S, int32_t batch,
                  int32_t loss_kind, double op_c0, double* loss) {
  return nguard(h, [&] {
    if (!x || !t || ncrops <= 0 || batch <= 0 || !loss) throw std::runtime_error("bad evaluation arguments");
    h->n.check(batch, S, S, false);
    double se = 0.0, st2 = 0.0;
    for (long long c0 = 0; c0 < ncrops; c0 += batch) {
      int b = (int)std::min<long long>(batch, ncrops - c0);
      batch_loss(h, x, t, w, c0, b, S, loss_kind, (float)op_c0, &se, &st2);
    }
    *loss = se / std::max(st2, 1e-300);
    return VSAV_OK;
  });
}

}  // extern "C"
