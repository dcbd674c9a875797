// net_api.cu -- the C ABI of the learned coarse proposal's network object (include/optflow_cuda_net.h): float32
// parameters, Adam moments, the bfloat16 copy of the weights and a pool of work buffers on one device.
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "common.cuh"
#include "net.cuh"
#include "../../include/optflow_cuda_net.h"

namespace {

// named device buffers, grown on demand (a grown buffer is freed once the device has finished with it)
struct Pool {
  std::map<std::string, std::pair<void*, size_t>> bufs;
  void* get(const std::string& name, size_t bytes) {
    auto it = bufs.find(name);
    if (it != bufs.end() && it->second.second >= bytes) return it->second.first;
    if (it != bufs.end()) {
      OFC_CUDA(cudaDeviceSynchronize());
      OFC_CUDA(cudaFree(it->second.first));
      bufs.erase(it);
    }
    void* p = nullptr;
    OFC_CUDA(cudaMalloc(&p, bytes));
    bufs[name] = {p, bytes};
    return p;
  }
  ~Pool() {
    for (auto& kv : bufs) cudaFree(kv.second.first);
  }
};

void set_err(char* err, size_t len, const std::string& m) {
  if (err && len) {
    size_t n = std::min(len - 1, m.size());
    std::memcpy(err, m.data(), n);
    err[n] = 0;
  }
}

}  // namespace

struct ofc_net {
  int device = 0;
  std::mutex mu;
  Pool pool;
  float* params = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* grads = nullptr;
  uint16_t* w16 = nullptr;
  double* dloss = nullptr;
  int step = 0;
};

namespace {

template <class F>
int net_guarded(ofc_net* n, char* err, size_t errlen, F&& f) {
  if (!n) {
    set_err(err, errlen, "null network");
    return OFC_ERR_ARG;
  }
  std::unique_lock<std::mutex> lk(n->mu, std::try_to_lock);
  if (!lk.owns_lock()) {
    set_err(err, errlen, "the network is busy: one call at a time");
    return OFC_ERR_BUSY;
  }
  try {
    OFC_CUDA(cudaSetDevice(n->device));
    f();
    return OFC_OK;
  } catch (const ofc::Error& x) {
    set_err(err, errlen, x.what());
    return x.status;
  } catch (const std::exception& x) {
    set_err(err, errlen, x.what());
    return OFC_ERR_DEVICE;
  }
}

ofc::net::Workspace workspace(ofc_net* n, void* stream) {
  return {[n](const std::string& name, size_t bytes) { return n->pool.get(name, bytes); }, (cudaStream_t)stream};
}

}  // namespace

extern "C" {

size_t ofc_net_param_count(void) { return ofc::net::param_count(); }

ofc_net* ofc_net_create(int device, char* err, size_t errlen) {
  ofc_net* n = new ofc_net();
  n->device = device;
  int st = net_guarded(n, err, errlen, [&] {
    const size_t P = ofc::net::param_count();
    n->params = (float*)n->pool.get("params", P * 4);
    n->m = (float*)n->pool.get("adam_m", P * 4);
    n->v = (float*)n->pool.get("adam_v", P * 4);
    n->grads = (float*)n->pool.get("grads", P * 4);
    n->w16 = (uint16_t*)n->pool.get("w16", P * 2);
    n->dloss = (double*)n->pool.get("loss", 8);
    OFC_CUDA(cudaMemset(n->params, 0, P * 4));
    OFC_CUDA(cudaMemset(n->m, 0, P * 4));
    OFC_CUDA(cudaMemset(n->v, 0, P * 4));
    OFC_CUDA(cudaMemset(n->w16, 0, P * 2));
  });
  if (st != OFC_OK) {
    delete n;
    return nullptr;
  }
  return n;
}

void ofc_net_destroy(ofc_net* n) {
  if (!n) return;
  cudaSetDevice(n->device);
  cudaDeviceSynchronize();
  delete n;
}

int ofc_net_set_params(ofc_net* n, const float* params, size_t cnt, char* err, size_t errlen) {
  return net_guarded(n, err, errlen, [&] {
    const size_t P = ofc::net::param_count();
    if (!params || cnt != P) throw ofc::Error(OFC_ERR_ARG, "expected " + std::to_string(P) + " parameters");
    OFC_CUDA(cudaDeviceSynchronize());
    OFC_CUDA(cudaMemcpy(n->params, params, P * 4, cudaMemcpyHostToDevice));
    OFC_CUDA(cudaMemset(n->m, 0, P * 4));
    OFC_CUDA(cudaMemset(n->v, 0, P * 4));
    n->step = 0;
    ofc::net::to_bf16(workspace(n, nullptr), n->params, n->w16);
    OFC_CUDA(cudaDeviceSynchronize());
  });
}

int ofc_net_get_params(ofc_net* n, float* params, size_t cnt, char* err, size_t errlen) {
  return net_guarded(n, err, errlen, [&] {
    const size_t P = ofc::net::param_count();
    if (!params || cnt != P) throw ofc::Error(OFC_ERR_ARG, "expected room for " + std::to_string(P) + " parameters");
    OFC_CUDA(cudaDeviceSynchronize());
    OFC_CUDA(cudaMemcpy(params, n->params, P * 4, cudaMemcpyDeviceToHost));
  });
}

int ofc_net_forward(ofc_net* n, const float* i1, const float* i2, int nb, int h, int w, float* flow, void* stream,
                    char* err, size_t errlen) {
  return net_guarded(n, err, errlen, [&] {
    if (!i1 || !i2 || !flow || nb < 1) throw ofc::Error(OFC_ERR_ARG, "null buffer or empty batch");
    ofc::net::forward(workspace(n, stream), n->params, n->w16, i1, i2, nb, h, w, flow);
  });
}

int ofc_net_gradients(ofc_net* n, const float* i1, const float* i2, int nb, int h, int w, const float* target,
                      const uint8_t* mask, float* flow, float* grads, double* loss, void* stream, char* err,
                      size_t errlen) {
  return net_guarded(n, err, errlen, [&] {
    if (!i1 || !i2 || !target || !mask || !flow || nb < 1) throw ofc::Error(OFC_ERR_ARG, "null buffer or empty batch");
    ofc::net::forward_backward(workspace(n, stream), n->params, n->w16, i1, i2, nb, h, w, target, mask, flow,
                               grads ? grads : n->grads, n->dloss);
    if (loss) {
      OFC_CUDA(cudaMemcpyAsync(loss, n->dloss, sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
      OFC_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    }
  });
}

int ofc_net_adam(ofc_net* n, const float* grads, float lr, void* stream, char* err, size_t errlen) {
  return net_guarded(n, err, errlen, [&] {
    n->step++;
    ofc::net::adam(workspace(n, stream), n->params, grads ? grads : n->grads, n->m, n->v, n->w16, lr, 0.9f, 0.999f,
                   1e-8f, n->step);
  });
}

}  // extern "C"
