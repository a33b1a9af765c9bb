// C ABI of the learned-closure MLP (include/hit3d.h): inference and the
// loss gradients of one training batch.  Training runs the fused k_mlp pass
// (forward, loss gradient, backward through the layers) and then the four
// weight-gradient GEMMs dW_l = a_{l-1}^T dz_l over the batch on the tensor
// cores, split along the points.
#include <string>

#include "hit3d.h"
#include "kernels.h"

namespace hit {
int record_error(int code, const std::string& msg);
}

namespace {
using hit::MlpArgs;

constexpr int MLP_GRID = 2 * 148;  // two 75 KB CTAs (256 TMEM columns each) per SM
constexpr int GRAD_SPLITS = 296;
constexpr long long ROWS = 16 + 3 * 65 + 3 * 64 + 16;  // feature-major rows of the workspace

__global__ void k_loss(const double* part, int n, double scale, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += part[i];
    *out = s * scale;
  }
}

int cuda_err(cudaError_t e, const char* what) {
  return hit::record_error(HIT_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

bool weights_ok(const hit_mlp_weights* w, bool train) {
  if (!w || !w->w1t || !w->w2t || !w->w3t || !w->w4t || !w->b2 || !w->b3 || !w->b4) return false;
  return !train || (w->w2 && w->w3 && w->w4);
}

MlpArgs args_of(const hit_mlp_weights* w) {
  MlpArgs a{};
  a.w1t = static_cast<const __nv_bfloat16*>(w->w1t);
  a.w2t = static_cast<const __nv_bfloat16*>(w->w2t);
  a.w3t = static_cast<const __nv_bfloat16*>(w->w3t);
  a.w4t = static_cast<const __nv_bfloat16*>(w->w4t);
  a.w2 = static_cast<const __nv_bfloat16*>(w->w2);
  a.w3 = static_cast<const __nv_bfloat16*>(w->w3);
  a.w4 = static_cast<const __nv_bfloat16*>(w->w4);
  a.b2 = w->b2;
  a.b3 = w->b3;
  a.b4 = w->b4;
  return a;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// One fused k_mlp pass over P points (forward, output cotangent, backward
// through the layers; a.tau or a.ybar set) and the four weight-gradient GEMMs
// dW_l = a_{l-1}^T dz_l; loss (nullable) receives the MSE loss.
int run_grads(MlpArgs a, int64_t P, void* ws, float* dW1, float* dW2, float* dW3, float* dW4, double* loss, int* err,
              cudaStream_t st, const char* who) {
  if (P < 16 || P % 16) return hit::record_error(HIT_E_INVALID, std::string(who) + ": P must be a positive multiple of 16");
  if (P > (int64_t)1 << 30) return hit::record_error(HIT_E_UNSUPPORTED, std::string(who) + ": P too large");
  a.P = P;
  a.inv_count = (float)(1.0 / ((double)P * 6.0));
  a.err = err;
  __nv_bfloat16* b = static_cast<__nv_bfloat16*>(ws);
  auto take = [&](int rows) {
    __nv_bfloat16* r = b;
    b += (size_t)rows * P;
    return r;
  };
  a.aT0 = take(16);
  a.aT1 = take(65);
  a.aT2 = take(65);
  a.aT3 = take(65);
  a.dzT1 = take(64);
  a.dzT2 = take(64);
  a.dzT3 = take(64);
  a.dzT4 = take(16);
  unsigned char* rest = static_cast<unsigned char*>(ws) + align256((size_t)ROWS * P * 2);
  float* work = reinterpret_cast<float*>(rest);
  double* part = reinterpret_cast<double*>(rest + align256((size_t)GRAD_SPLITS * 65 * 64 * 4));
  a.loss = part;
  const int grid = (int)std::min<int64_t>((P + 127) / 128, MLP_GRID);
  cudaError_t e = hit::launch_mlp(a, grid, st);
  if (e != cudaSuccess) return cuda_err(e, who);
  const int K = (int)P, splits = (int)std::min<int64_t>(GRAD_SPLITS, P / 16);
  struct G {
    const __nv_bfloat16 *A, *B;
    float* C;
    int M, N;
  } gs[4] = {{a.aT3, a.dzT4, dW4, 65, 16}, {a.aT2, a.dzT3, dW3, 65, 64}, {a.aT1, a.dzT2, dW2, 65, 64},
             {a.aT0, a.dzT1, dW1, 16, 64}};
  for (const G& g : gs) {
    e = hit::launch_tcgemm(g.A, K, g.B, K, g.C, g.N, g.M, g.N, K, err, st, splits, work);
    if (e != cudaSuccess) return cuda_err(e, who);
  }
  if (!loss) return HIT_OK;
  k_loss<<<1, 32, 0, st>>>(part, grid, 1.0 / ((double)P * 6.0), loss);
  e = cudaGetLastError();
  return e == cudaSuccess ? HIT_OK : cuda_err(e, who);
}
}  // namespace

extern "C" {

int hit_mlp_forward_strided(const hit_mlp_weights* w, const float* x, int64_t x_sf, int64_t x_sp, int64_t P, float* y,
                            int64_t y_sf, int64_t y_sp, int ctas_per_sm, int* err, void* stream) {
  if (!weights_ok(w, false) || !x || !y || !err) return hit::record_error(HIT_E_INVALID, "mlp_forward: NULL argument");
  if (P < 1) return hit::record_error(HIT_E_INVALID, "mlp_forward: P must be >= 1");
  if (ctas_per_sm < 0) return hit::record_error(HIT_E_INVALID, "mlp_forward: ctas_per_sm must be >= 0");
  MlpArgs a = args_of(w);
  a.x = x;
  a.y = y;
  a.P = P;
  a.x_sf = x_sf;
  a.x_sp = x_sp;
  a.y_sf = y_sf;
  a.y_sp = y_sp;
  a.err = err;
  // one resident wave of inference CTAs, or ctas_per_sm of them per SM
  cudaError_t e = hit::launch_mlp(a, -ctas_per_sm, (cudaStream_t)stream);
  return e == cudaSuccess ? HIT_OK : cuda_err(e, "mlp_forward");
}

int hit_mlp_forward(const hit_mlp_weights* w, const float* x, int64_t P, float* y, int* err, void* stream) {
  return hit_mlp_forward_strided(w, x, 1, 9, P, y, 1, 6, 0, err, stream);
}

int64_t hit_mlp_workspace_bytes(int64_t P) {
  if (P < 1) return 0;
  return (int64_t)(align256((size_t)ROWS * P * 2) + align256((size_t)GRAD_SPLITS * 65 * 64 * 4) +
                   align256(MLP_GRID * sizeof(double)));
}

int hit_mlp_train_grads(const hit_mlp_weights* w, const float* x, const float* tau, int64_t P, void* ws, float* dW1,
                        float* dW2, float* dW3, float* dW4, double* loss, int* err, void* stream) {
  if (!weights_ok(w, true) || !x || !tau || !ws || !dW1 || !dW2 || !dW3 || !dW4 || !loss || !err)
    return hit::record_error(HIT_E_INVALID, "mlp_train_grads: NULL argument");
  MlpArgs a = args_of(w);
  a.x = x;
  a.x_sf = 1;
  a.x_sp = 9;
  a.tau = tau;
  return run_grads(a, P, ws, dW1, dW2, dW3, dW4, loss, err, (cudaStream_t)stream, "mlp_train_grads");
}

int hit_mlp_vjp(const hit_mlp_weights* w, const void* w1, const float* x, int64_t x_sf, int64_t x_sp,
                const float* ybar, int64_t y_sf, int64_t y_sp, int64_t P, void* ws, float* dW1, float* dW2,
                float* dW3, float* dW4, float* xbar, int* err, void* stream) {
  if (!weights_ok(w, true) || !x || !ybar || !ws || !dW1 || !dW2 || !dW3 || !dW4 || !err || (xbar && !w1))
    return hit::record_error(HIT_E_INVALID, "mlp_vjp: NULL argument");
  MlpArgs a = args_of(w);
  a.x = x;
  a.x_sf = x_sf;
  a.x_sp = x_sp;
  a.tau = ybar;  // selects the training instantiation; the cotangent replaces the loss gradient
  a.ybar = ybar;
  a.yb_sf = y_sf;
  a.yb_sp = y_sp;
  a.xbar = xbar;
  a.w1 = static_cast<const __nv_bfloat16*>(w1);
  return run_grads(a, P, ws, dW1, dW2, dW3, dW4, nullptr, err, (cudaStream_t)stream, "mlp_vjp");
}

}  // extern "C"
