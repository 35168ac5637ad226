// mlp_oracle.cpp -- CPU ORACLE (test infrastructure only): C entry points of
// the FP64 multilayer perceptron in mlp_oracle.h, for the tests' ctypes
// bindings (oracle/oracle.py).
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "mlp_oracle.h"

extern "C" {

int orc_mlp_nparam() { return orc::kNParam; }

// Y[n][6] = mlp(X[n][11]) on normalised inputs/outputs.
void orc_mlp_forward(const double* P, const double* X, long long n, double* Y, int bf16) {
#pragma omp parallel for schedule(static)
  for (long long s = 0; s < n; s++) {
    orc::MlpTrace t;
    orc::mlp_forward(P, X + s * orc::kIn, t, bf16 != 0);
    for (int o = 0; o < orc::kOut; o++) Y[s * orc::kOut + o] = t.y[o];
  }
}

// Mean-squared-error loss over n samples and its gradient G[9478].
double orc_mlp_loss_grad(const double* P, const double* X, const double* Y, long long n, double* G) {
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  std::vector<std::vector<double>> Gt(nt, std::vector<double>(orc::kNParam, 0.0));
  std::vector<double> lt(nt, 0.0);
  const double inv = 1.0 / ((double)n * orc::kOut);
#pragma omp parallel
  {
    int id = 0;
#ifdef _OPENMP
    id = omp_get_thread_num();
#endif
    orc::MlpTrace t;
#pragma omp for schedule(static)
    for (long long s = 0; s < n; s++) {
      orc::mlp_forward(P, X + s * orc::kIn, t, false);
      lt[id] += orc::mlp_backward(P, t, Y + s * orc::kOut, inv, Gt[id].data());
    }
  }
  double loss = 0.0;
  for (int i = 0; i < orc::kNParam; i++) G[i] = 0.0;
  for (int k = 0; k < nt; k++) {
    loss += lt[k];
    for (int i = 0; i < orc::kNParam; i++) G[i] += Gt[k][i];
  }
  return loss;
}

double orc_mlp_loss(const double* P, const double* X, const double* Y, long long n) {
  return orc::mlp_loss(P, X, Y, n);
}

void orc_mlp_adam(double* P, double* m, double* v, const double* g, int n, double lr, double b1, double b2,
                  double eps, int step) {
  orc::adam_update(P, m, v, g, n, lr, b1, b2, eps, step);
}

double orc_bf16_round(double v) { return orc::bf16_round(v); }

}  // extern "C"
