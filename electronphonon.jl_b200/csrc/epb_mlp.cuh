// The learned surrogate's state, shared by its FP32 (epb_mlp.cu) and tensor-core (epb_mlp_tc.cu) kernels.
#pragma once

#include <vector>

#include "epb_common.cuh"

struct epb_mlp {
  epb_ctx* ctx = nullptr;
  int nf = 0, nin = 0, hidden = 0, nhidden = 0, nout = 0;
  int64_t nparam = 0;
  std::vector<int64_t> w_off, b_off;  // per linear layer
  std::vector<int> fan_in, fan_out;
  int4* fvec = nullptr;     // feature vectors (device)
  float* params = nullptr;  // [nparam]
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* y_mu = nullptr;    // [nout]
  float* y_sc = nullptr;    // [nout]
  double* margin = nullptr;  // [nout] calibrated culling margin (Ry)
  std::vector<double> margin_host;
  bool scaled = false;
  bool calibrated = false;
  int64_t* step = nullptr;  // device step counter (Adam t)
  double* loss_acc = nullptr;  // device per-epoch loss sums (grown on demand)
  int64_t loss_cap = 0;
  // inference: 1 = BF16 tensor cores (tcgen05) when the shape allows it, 0 = FP32 SGEMM kernels
  int infer_mode = 1;
  uint8_t* tc_image = nullptr;  // BF16 weights in the swizzled K-major shared-memory image, per layer
  bool tc_dirty = true;         // parameters changed since the image was built
};

