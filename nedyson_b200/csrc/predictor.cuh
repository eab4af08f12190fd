// Learned next-step predictor (see predictor.cu).
#pragma once
#include "engine.cuh"
#include <cuda_bf16.h>

namespace nedy {

constexpr int PRED_IN = 12, PRED_W = 256;
constexpr long long PRED_NPARAM = (long long)PRED_W * PRED_IN + PRED_W + (long long)PRED_W * PRED_W + PRED_W +
                                  2LL * PRED_W + 2;

class Predictor {
 public:
  Predictor(Ctx &c, i64 capacity, unsigned long long seed);
  ~Predictor();
  void init(unsigned long long seed);
  void set_params(const float *host);
  void get_params(float *host);
  // training samples of the converged row T (every stride-th eligible element, hashed)
  void collect(const DevGF &g, int T, int stride);
  i64 samples();
  void clear_samples();
  double train(int iters, int batch, double lr);
  // adds the learned correction to row T (which holds the polynomial extrapolation);
  // corr_out (optional, row_elements values) receives the corrections
  void apply(const DevGF &g, int T, double2 *corr_out);
  // the network on the tensor cores for n given input rows (device x: n x PRED_IN, y: n x 2)
  void infer(int n, const float *x, float *y);
  static i64 row_elements(const DevGF &g, int T);
  // after the first corrector iteration: max change from the learned and from the plain
  // prediction over the corrected elements (saved: the row before the iteration)
  void judge(const DevGF &g, int T, const double2 *saved, const double2 *corr, double &d_learned, double &d_plain);
  // loss and gradient (into the device gradient buffer) on B rows already on the device
  double loss_grad(int B, const float *xb, const float *tb, bool want_loss);
  void forward(int B, const float *xb, float *h1, float *h2, float *y);
  const float *grad() const { return G; }

  Ctx &ctx;
  i64 cap;
  unsigned long long seed;

 private:
  void ensure_work(int B);
  float *W = nullptr, *G = nullptr, *Mo = nullptr, *Vo = nullptr;
  float *X = nullptr, *Y = nullptr;
  unsigned long long *count = nullptr;  // sample count, loss (double), two judge words
  double *dloss = nullptr;
  float *work = nullptr;
  i64 work_cap = 0;
  unsigned long long ncollect = 0;
  long long adam_t = 0;
  // selection of the elements the network corrects (grown once for the longest row)
  double *s6buf = nullptr;
  i64 *sel = nullptr;
  unsigned long long *selw = nullptr;  // [0] row max of s6 (as bits), [1] selected count, then the error word
  i64 sel_cap = 0;
  void ensure_mlp();
  int *err_word() const;
  void check_err();
};

}  // namespace nedy
