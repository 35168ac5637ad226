// mlp_oracle.h -- CPU ORACLE (test infrastructure only): the learned SGS
// closure's multilayer perceptron in FP64.
//
// The closure has no counterpart in the reference (it replaces the eddy
// viscosity of complen.f90:1-28 and the stresses of compsgs1.f90:1-53
// with a network); this file is the checker for the product's tensor-core
// kernels and for the solver's learned stage.
//
// Network: 11 -> 64 -> 64 -> 64 -> 6, GELU (tanh form) after each hidden
// layer, identity output.  Inputs and outputs are normalised:
//   x_j = (f_j - in_shift_j) * in_scale_j,    tau_i = y_i * out_scale_i + out_shift_i
// Features f (in this order): the nine velocity gradients d_i u_j times the
// filter width Delta, i.e. (ux, vx, wx, uy, vy, wy, uz, vz, wz) * Delta,
// then z+ = z_wall * Re_tau / h, then Delta.  Outputs: tau11, tau22, tau33,
// tau12, tau13, tau23.
//
// Flat parameter vector (float / double, 9478 values):
//   W1[64][11], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], W4[6][64], b4[6]
// Normalisation vector (34 values): in_shift[11], in_scale[11],
//   out_scale[6], out_shift[6].
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

constexpr int kIn = 11, kHid = 64, kOut = 6;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kHid, kOffW4 = kOffB3 + kHid,
              kOffB4 = kOffW4 + kOut * kHid, kNParam = kOffB4 + kOut;
static_assert(kNParam == 9478, "parameter count");
constexpr int kNNorm = 2 * kIn + 2 * kOut;

// round-to-nearest-even to bfloat16, returned as double
inline double bf16_round(double v) {
  float f = (float)v;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (double)f;  // inf / nan unchanged
  uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  u &= 0xffff0000u;
  std::memcpy(&f, &u, 4);
  return (double)f;
}

constexpr double kGeluC = 0.7978845608028654;  // sqrt(2/pi)
constexpr double kGeluA = 0.044715;
inline double gelu(double z) { return 0.5 * z * (1.0 + std::tanh(kGeluC * (z + kGeluA * z * z * z))); }
inline double gelu_d(double z) {
  double t = std::tanh(kGeluC * (z + kGeluA * z * z * z));
  return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * kGeluC * (1.0 + 3.0 * kGeluA * z * z);
}

// Forward pass of one sample; the pre-activations z1..z3 and activations
// a1..a3 are kept for the backward pass.  bf16 = true rounds the inputs,
// weights and hidden activations to bfloat16 (the product's storage types);
// sums stay FP64.
struct MlpTrace {
  double x[kIn], z1[kHid], a1[kHid], z2[kHid], a2[kHid], z3[kHid], a3[kHid], y[kOut];
};

inline void mlp_forward(const double* P, const double* x, MlpTrace& t, bool bf16) {
  auto q = [&](double v) { return bf16 ? bf16_round(v) : v; };
  for (int i = 0; i < kIn; i++) t.x[i] = q(x[i]);
  auto layer = [&](const double* W, const double* b, const double* in, int nin, double* z, double* a, int nout,
                   bool act) {
    for (int o = 0; o < nout; o++) {
      double s = 0.0;
      for (int i = 0; i < nin; i++) s += q(W[o * nin + i]) * in[i];
      z[o] = s + b[o];
      if (act) a[o] = q(gelu(z[o]));
    }
  };
  layer(P + kOffW1, P + kOffB1, t.x, kIn, t.z1, t.a1, kHid, true);
  layer(P + kOffW2, P + kOffB2, t.a1, kHid, t.z2, t.a2, kHid, true);
  layer(P + kOffW3, P + kOffB3, t.a2, kHid, t.z3, t.a3, kHid, true);
  layer(P + kOffW4, P + kOffB4, t.a3, kHid, t.y, nullptr, kOut, false);
}

// Loss L = sum over samples and outputs of (y - target)^2 / (n * 6).
// Accumulates dL/dP for one sample (with the 1/(n*6) factor) into G.
inline double mlp_backward(const double* P, const MlpTrace& t, const double* target, double inv_count, double* G) {
  double dy[kOut], loss = 0.0;
  for (int o = 0; o < kOut; o++) {
    double r = t.y[o] - target[o];
    loss += r * r;
    dy[o] = 2.0 * r * inv_count;
  }
  // layer 4
  double da3[kHid] = {0};
  for (int o = 0; o < kOut; o++) {
    G[kOffB4 + o] += dy[o];
    for (int i = 0; i < kHid; i++) {
      G[kOffW4 + o * kHid + i] += dy[o] * t.a3[i];
      da3[i] += dy[o] * P[kOffW4 + o * kHid + i];
    }
  }
  auto back = [&](const double* W, int offW, int offB, const double* z, const double* da, const double* in, int nin,
                  double* din) {
    for (int i = 0; i < nin && din; i++) din[i] = 0.0;
    for (int o = 0; o < kHid; o++) {
      double dz = da[o] * gelu_d(z[o]);
      G[offB + o] += dz;
      for (int i = 0; i < nin; i++) {
        G[offW + o * nin + i] += dz * in[i];
        if (din) din[i] += dz * W[o * nin + i];
      }
    }
  };
  double da2[kHid], da1[kHid];
  back(P + kOffW3, kOffW3, kOffB3, t.z3, da3, t.a2, kHid, da2);
  back(P + kOffW2, kOffW2, kOffB2, t.z2, da2, t.a1, kHid, da1);
  back(P + kOffW1, kOffW1, kOffB1, t.z1, da1, t.x, kIn, nullptr);
  return loss * inv_count;
}

// Batch loss and gradient (G overwritten).
inline double mlp_loss_grad(const double* P, const double* X, const double* Y, long long n, double* G) {
  std::memset(G, 0, sizeof(double) * kNParam);
  double inv = 1.0 / ((double)n * kOut), loss = 0.0;
  MlpTrace t;
  for (long long s = 0; s < n; s++) {
    mlp_forward(P, X + s * kIn, t, false);
    loss += mlp_backward(P, t, Y + s * kOut, inv, G);
  }
  return loss;
}

inline double mlp_loss(const double* P, const double* X, const double* Y, long long n) {
  double inv = 1.0 / ((double)n * kOut), loss = 0.0;
  MlpTrace t;
  for (long long s = 0; s < n; s++) {
    mlp_forward(P, X + s * kIn, t, false);
    for (int o = 0; o < kOut; o++) {
      double r = t.y[o] - Y[s * kOut + o];
      loss += r * r;
    }
  }
  return loss * inv;
}

// Adam (Kingma & Ba 2015) with bias correction; step counts from 1.
inline void adam_update(double* P, double* m, double* v, const double* g, int n, double lr, double b1, double b2,
                        double eps, int step) {
  double c1 = 1.0 - std::pow(b1, step), c2 = 1.0 - std::pow(b2, step);
  for (int i = 0; i < n; i++) {
    m[i] = b1 * m[i] + (1.0 - b1) * g[i];
    v[i] = b2 * v[i] + (1.0 - b2) * g[i] * g[i];
    double mh = m[i] / c1, vh = v[i] / c2;
    P[i] -= lr * mh / (std::sqrt(vh) + eps);
  }
}

}  // namespace orc
