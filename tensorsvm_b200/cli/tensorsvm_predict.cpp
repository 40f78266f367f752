// tensorsvm-predict: labels of a LIBSVM test file under a tensorsvm-train model file.
//
// The reference leaves prediction to ThunderSVM (README.md:27-31) and its own predict
// (tensorsvm-train.cu:166-270) is never called.  This follows svm-predict's command line
// (test_file model_file output_file; one predicted label per output line; the accuracy line
// when the test file carries labels) over the library: tsvm_read_model, tsvm_read_libsvm and
// tsvm_predict (decision values on the GPU).
//   -dec : write "label decision_value" per line instead of the label alone
//   -q   : no accuracy line
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "tensorsvm.h"

int main(int argc, char **argv) {
  bool dec = false, quiet = false;
  const char *paths[3] = {nullptr, nullptr, nullptr};
  int np = 0;
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "-dec")) dec = true;
    else if (!strcmp(argv[i], "-q")) quiet = true;
    else if (np < 3) paths[np++] = argv[i];
    else np = 4;
  }
  if (np != 3) {
    printf("Usage: tensorsvm-predict [-dec] [-q] test_file model_file output_file\n");
    return 1;
  }
  const auto t0 = std::chrono::steady_clock::now();
  tsvm_model_view m{};
  int pos = 0, neg = 0;
  tsvm_status st = tsvm_read_model(paths[1], &m, &pos, &neg);
  if (st != TSVM_OK) {
    fprintf(stderr, "can't read model file %s: %s\n", paths[1], tsvm_status_string(st));
    return 1;
  }
  float *L = nullptr, *X = nullptr;
  int64_t n = 0, d = 0, nnz = 0, bad = 0;
  st = tsvm_read_libsvm(paths[0], 0, 0, &L, &X, &n, &d, &nnz, &bad);
  if (st != TSVM_OK) {
    if (bad > 0) fprintf(stderr, "Wrong input format at line %lld\n", (long long)bad);
    else fprintf(stderr, "can't open test file %s\n", paths[0]);
    tsvm_free_model(&m);
    return 1;
  }
  // common width: features beyond the model's (or the file's) last index are zero there
  const int64_t dd = std::max<int64_t>(d, m.d);
  std::vector<float> T;
  const float *rows = X;
  if (dd != d) {
    T.assign((size_t)n * dd, 0.f);
    for (int64_t i = 0; i < n; ++i)
      std::copy(X + (size_t)i * d, X + (size_t)(i + 1) * d, T.begin() + (size_t)i * dd);
    rows = T.data();
  }
  std::vector<float> S;
  tsvm_model_view mv = m;
  if (dd != m.d) {
    const int64_t rows_sv = m.kernel == TSVM_KERNEL_RBF ? m.nsv : 1;
    S.assign((size_t)rows_sv * dd, 0.f);
    for (int64_t i = 0; i < rows_sv; ++i)
      std::copy(m.sv + (size_t)i * m.d, m.sv + (size_t)(i + 1) * m.d, S.begin() + (size_t)i * dd);
    mv.sv = S.data();
  }
  mv.d = (int32_t)dd;
  tsvm_context *ctx = nullptr;
  st = tsvm_create(&ctx, 0);
  std::vector<double> f((size_t)n);
  if (st == TSVM_OK) st = tsvm_predict(ctx, &mv, rows, n, f.data());
  if (ctx) tsvm_destroy(ctx);
  if (st != TSVM_OK) {
    fprintf(stderr, "tensorsvm: %s\n", tsvm_status_string(st));
    tsvm_free(L);
    tsvm_free(X);
    tsvm_free_model(&m);
    return 1;
  }
  FILE *out = fopen(paths[2], "w");
  if (!out) {
    fprintf(stderr, "can't open output file %s\n", paths[2]);
    return 1;
  }
  int64_t correct = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int lab = f[i] > 0 ? pos : neg;
    if (lab == (int)L[i]) ++correct;
    if (dec) fprintf(out, "%d %.17g\n", lab, f[i]);
    else fprintf(out, "%d\n", lab);
  }
  fclose(out);
  if (!quiet)
    printf("Accuracy = %g%% (%lld/%lld) (classification)\n", n ? 100.0 * correct / n : 0.0,
           (long long)correct, (long long)n);
  if (!quiet)
    printf("predict elapsed time = %.4f seconds\n",
           std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  tsvm_free(L);
  tsvm_free(X);
  tsvm_free_model(&m);
  return 0;
}
