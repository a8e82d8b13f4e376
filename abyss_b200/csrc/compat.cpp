// Reference-compatible drop-in (include/abyss_reg_compat.h): the six entry
// points of src_mpi/cuda/cuda_functions.h:3-10 and their FP64 spelling from
// src/cuda/cuda_functions.h:3-10, implemented on the context API.
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "../../include/abyss_reg.h"
#include "../../include/abyss_reg_compat.h"
#include <cuda_runtime.h>
#include <chrono>

namespace {

struct CompatState {
  std::mutex mu;
  abyss_ctx *ctx = nullptr;
  bool is_open = false;
  int stride = 1000;  // NumNeighborMax, src_mpi/def.h:20
  int status = ABYSS_OK;
  int nnb_last = 0;   // NNB of the last SendToDevice
  // profile counters (the reference's time_send/time_grav, cuda_my_acceleration.cu:24)
  long long calls = 0, sends = 0, targets = 0;
  double pairs = 0.0, t_send = 0.0, t_grav = 0.0;
  std::vector<double> acc, jerk;
  std::vector<int> list;
};

CompatState &st() {
  static CompatState s;
  return s;
}

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int ensure_ctx(CompatState &s, int irank) {
  if (s.ctx) return ABYSS_OK;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return ABYSS_ERR_NODEVICE;
  int dev = irank >= 0 ? irank % count : 0;
  if (const char *e = std::getenv("ABYSS_DEVICE")) dev = std::atoi(e) % count;
  return abyss_create(dev, &s.ctx);
}

template <class T>
void send_impl(int *NNB, T m[], T x[][3], T v[][3], T r2[]) {
  CompatState &s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  const double t0 = now_s();
  if (!NNB || *NNB <= 0 || !m || !x || !v || !r2) {
    std::fprintf(stderr, "abyss: SendToDevice: bad arguments\n");
    s.status = ABYSS_ERR_ARG;
    return;
  }
  int rc = ensure_ctx(s, 0);
  if (rc != ABYSS_OK) {
    std::fprintf(stderr, "abyss: SendToDevice: no CUDA device\n");
    s.status = rc;
    return;
  }
  const int n = *NNB;
  std::vector<double> px(3 * (size_t)n), pv(3 * (size_t)n), mm(n), rr(n);
  for (int j = 0; j < n; ++j) {
    for (int d = 0; d < 3; ++d) {
      px[3 * (size_t)j + d] = (double)x[j][d];
      pv[3 * (size_t)j + d] = (double)v[j][d];
    }
    mm[j] = (double)m[j];
    rr[j] = (double)r2[j];
  }
  rc = abyss_upload_predicted(s.ctx, n, px.data(), pv.data(), mm.data(), rr.data());
  if (rc == ABYSS_OK) rc = abyss_synchronize(s.ctx);
  if (rc != ABYSS_OK) std::fprintf(stderr, "abyss: SendToDevice: %s\n", abyss_last_error(s.ctx));
  s.status = rc;
  s.nnb_last = n;
  s.sends++;
  s.t_send += now_s() - t0;
}

template <class T>
void calc_impl(int *NumTarget, int *h_target_list, T acc[][3], T adot[][3], int NumNeighbor[],
               int *NeighborList) {
  CompatState &s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  const double t0 = now_s();
  if (!s.ctx || s.nnb_last <= 0) {
    std::fprintf(stderr, "abyss: CalculateAccelerationOnDevice before SendToDevice\n");
    s.status = ABYSS_ERR_STATE;
    return;
  }
  if (!NumTarget || *NumTarget <= 0 || *NumTarget > s.nnb_last || !h_target_list || !acc || !adot ||
      !NumNeighbor || !NeighborList) {
    // the reference asserts 0 < NumTarget <= NNB (cuda_my_acceleration.cu:104)
    std::fprintf(stderr, "abyss: CalculateAccelerationOnDevice: bad arguments\n");
    s.status = ABYSS_ERR_ARG;
    return;
  }
  const int m = *NumTarget;
  s.acc.resize(3 * (size_t)m);
  s.jerk.resize(3 * (size_t)m);
  s.list.resize((size_t)m * s.stride);
  int ovf = 0;
  int rc = abyss_regular_force(s.ctx, m, h_target_list, 0.0, s.stride, nullptr, s.acc.data(),
                               s.jerk.data(), nullptr, nullptr, NumNeighbor, s.list.data(), &ovf);
  if (rc < 0) {
    std::fprintf(stderr, "abyss: CalculateAccelerationOnDevice: %s\n", abyss_last_error(s.ctx));
    s.status = rc;
    return;
  }
  if (rc == ABYSS_WARN_OVERFLOW)
    std::fprintf(stderr, "abyss: %d targets have more than NumNeighborMax=%d neighbours; lists truncated\n",
                 ovf, s.stride);
  for (int i = 0; i < m; ++i) {
    for (int d = 0; d < 3; ++d) {
      acc[i][d] = (T)s.acc[3 * (size_t)i + d];
      adot[i][d] = (T)s.jerk[3 * (size_t)i + d];
    }
    const int k = NumNeighbor[i] < s.stride ? NumNeighbor[i] : s.stride;
    int *dst = NeighborList + (size_t)i * s.stride;
    const int *src = s.list.data() + (size_t)i * s.stride;
    for (int q = 0; q < k; ++q) dst[q] = src[q];
  }
  s.status = rc;
  s.calls++;
  s.targets += m;
  s.pairs += (double)m * (double)s.nnb_last;
  s.t_grav += now_s() - t0;
}

}  // namespace

extern "C" {

void InitializeDevice(int *irank) {
  CompatState &s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  const int r = irank ? *irank : 0;
  s.status = ensure_ctx(s, r);
  if (s.status != ABYSS_OK) std::fprintf(stderr, "abyss: InitializeDevice: no usable CUDA device\n");
}

void OpenDevice(const int *irank) {
  int r = irank ? *irank : 0;
  InitializeDevice(&r);
  CompatState &s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  if (s.is_open) {
    std::fprintf(stderr, "abyss: device is already open\n");  // cuda_my_acceleration.cu:895
    return;
  }
  s.is_open = true;
  s.calls = s.sends = s.targets = 0;
  s.pairs = s.t_send = s.t_grav = 0.0;
}

void CloseDevice(void) {
  CompatState &s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  if (!s.is_open) {
    std::fprintf(stderr, "abyss: device is already closed\n");  // cuda_my_acceleration.cu:907
    return;
  }
  s.is_open = false;
  if (s.ctx) abyss_destroy(s.ctx);
  s.ctx = nullptr;
  s.nnb_last = 0;
}

void ProfileDevice(int *irank) {
  CompatState &s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  if (std::getenv("ABYSS_PROFILE") && s.calls > 0) {
    // the reference's line at cuda_my_acceleration.cu:1040-1046 (60 flop per pair)
    std::fprintf(stderr,
                 "[R.%d GPU Reg.F] Nsend %lld Ngrav %lld <Ni> %lld send(s) %f grav(s) %f Perf.(Gflops) %f\n",
                 irank ? *irank : 0, s.sends, s.calls, s.targets / (s.calls ? s.calls : 1), s.t_send,
                 s.t_grav, 60e-9 * s.pairs / (s.t_grav > 0 ? s.t_grav : 1));
  }
  s.calls = s.sends = s.targets = 0;
  s.pairs = s.t_send = s.t_grav = 0.0;
}

void SendToDevice(int *NNB, float m[], float x[][3], float v[][3], float r2[], float mdot[]) {
  (void)mdot;
  send_impl<float>(NNB, m, x, v, r2);
}

void CalculateAccelerationOnDevice(int *NumTarget, int *h_target_list, float acc[][3],
                                   float adot[][3], int NumNeighbor[], int *NeighborList) {
  calc_impl<float>(NumTarget, h_target_list, acc, adot, NumNeighbor, NeighborList);
}

void SendToDevice_f64(int *NNB, double m[], double x[][3], double v[][3], double r2[],
                      double mdot[]) {
  (void)mdot;
  send_impl<double>(NNB, m, x, v, r2);
}

void CalculateAccelerationOnDevice_f64(int *NumTarget, int *h_target_list, double acc[][3],
                                       double adot[][3], int NumNeighbor[], int *NeighborList) {
  calc_impl<double>(NumTarget, h_target_list, acc, adot, NumNeighbor, NeighborList);
}

int abyss_compat_set_list_stride(int stride) {
  if (stride <= 0) return ABYSS_ERR_ARG;
  CompatState &s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  s.stride = stride;
  return ABYSS_OK;
}

int abyss_compat_status(void) {
  CompatState &s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  return s.status;
}

}  // extern "C"
