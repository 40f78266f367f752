// tensorsvm-train: the reference trainer's command line over libtensorsvm_b200.
//
// Same flags, defaults and positional rules as parsecmd (tensorsvm-train.cu:1099-1156), the
// same LIBSVM reader semantics (libsvmread, tensorsvm-train.cu:1162-1278), the same label
// remap (tensorsvm-train.cu:879-896) and the same model text (writemodel,
// tensorsvm-train.cu:273-417).  Deliberate differences, each an error the reference ignores:
//   * a malformed input line stops with a message and exit status 1 (the reference prints
//     "Wrong input format" and trains on partially read data);
//   * -t 2 with -g 0 uses gamma = 1/num_features, as the reference's help text documents
//     (the reference computes with gamma = 0);
//   * -s 1 (the reference's unimplemented PGD) exits with status 1 instead of writing an
//     uninitialised model.
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "tensorsvm.h"

namespace {

struct Args {
  int K = 50;          // tensorsvm-train.cu:66
  double C = 1;        // :67
  double g = 0;        // :68
  int T = 0;           // :69
  int S = 0;           // :70
  long NN = 0;         // -N
  const char *train = nullptr, *model = nullptr, *test = nullptr;
  bool analysis = false, tensorcore = false, scale256 = false, quiet = false;
  int precision = -1;  // -prec overrides -tensorcore
  double rel_gap = 0;  // -rel_gap (not in the reference)
  int max_iter = 100;
};

void help_msg() {
  printf("Usage: tensorsvm-train [options] training_set_file [model_file]\n"
         "options:\n"
         "-t kernel_type : 0 -- linear: u'*v (default)   2 -- radial basis function: exp(-gamma*|u-v|^2)\n"
         "-g gamma : set gamma in kernel function (default 1/num_features)\n"
         "-c cost : set the parameter C of C-SVC (default 1)\n"
         "-k rank : rank of the kernel factor (default 50)\n"
         "-s solver : 0 -- approx interior point method (default)\n"
         "-N n_samples : only consider the first n_samples in training\n"
         "-tensorcore : tensor-core (FP16, tcgen05) kernel-block products\n"
         "-prec fp32|bf16|fp16|bf16_fast|fp16_fast : contraction precision (overrides\n"
         "     -tensorcore); *_fast: one 16-bit product per factor pass, no hi+lo split\n"
         "-rel_gap tol : also stop at relative duality gap <= tol\n"
         "-scale256 : divide feature values by 256\n"
         "-analysis : report ||K||_F and ||K - Z Z'||_F (RBF, FP64 on the GPU)\n"
         "-test file : accuracy of the trained model on a LIBSVM test file\n"
         "-q : quiet\n");
}

bool parse(int argc, char **argv, Args &a) {
  bool have_train = false;
  for (int i = 1; i < argc; ++i) {
    auto next = [&](const char *flag) -> const char * {
      if (i + 1 >= argc) {
        fprintf(stderr, "Error: %s needs a value\n", flag);
        exit(1);
      }
      return argv[++i];
    };
    if (!strcmp(argv[i], "-c")) a.C = atof(next("-c"));
    else if (!strcmp(argv[i], "-g")) a.g = atof(next("-g"));
    else if (!strcmp(argv[i], "-test")) a.test = next("-test");
    else if (!strcmp(argv[i], "-t")) {
      a.T = atoi(next("-t"));
      if (a.T != 0 && a.T != 2) {
        printf("Error: unimplemented -t %d\n", a.T);
        exit(1);
      }
    } else if (!strcmp(argv[i], "-N")) a.NN = atol(next("-N"));
    else if (!strcmp(argv[i], "-k")) a.K = atoi(next("-k"));
    else if (!strcmp(argv[i], "-s")) a.S = atoi(next("-s"));
    else if (!strcmp(argv[i], "-analysis")) a.analysis = true;
    else if (!strcmp(argv[i], "-tensorcore")) a.tensorcore = true;
    else if (!strcmp(argv[i], "-scale256")) a.scale256 = true;
    else if (!strcmp(argv[i], "-q")) a.quiet = true;
    else if (!strcmp(argv[i], "-rel_gap")) a.rel_gap = atof(next("-rel_gap"));
    else if (!strcmp(argv[i], "-max_iter")) a.max_iter = atoi(next("-max_iter"));
    else if (!strcmp(argv[i], "-prec")) {
      const char *p = next("-prec");
      a.precision = !strcmp(p, "fp32") ? TSVM_PREC_FP32
                    : !strcmp(p, "bf16") ? TSVM_PREC_BF16
                    : !strcmp(p, "fp16") ? TSVM_PREC_FP16
                    : !strcmp(p, "bf16_fast") ? TSVM_PREC_BF16_FAST
                    : !strcmp(p, "fp16_fast") ? TSVM_PREC_FP16_FAST : -2;
      if (a.precision == -2) {
        fprintf(stderr, "Error: unknown precision %s\n", p);
        exit(1);
      }
    } else if (!have_train) {
      a.train = argv[i];
      have_train = true;
    } else {
      a.model = argv[i];
    }
  }
  return a.train != nullptr;
}

// LIBSVM reader of the library (tsvm_read_libsvm: parallel parse, the reference's index rules)
// with the reference's messages (tensorsvm-train.cu:1210-1211, 1236, 1245).
bool libsvm_read(const char *path, bool scale256, std::vector<float> &labels,
                 std::vector<float> &inst, long &n, long &nf) {
  float *L = nullptr, *M = nullptr;
  int64_t n64 = 0, d64 = 0, nnz = 0, bad = 0;
  const tsvm_status st = tsvm_read_libsvm(path, scale256 ? 1 : 0, 0, &L, &M, &n64, &d64, &nnz,
                                          &bad);
  if (st != TSVM_OK) {
    if (bad > 0) printf("Wrong input format at line %ld\n", (long)bad);
    else fprintf(stderr, "Can't open %s\n", path);
    return false;
  }
  n = (long)n64;
  nf = (long)d64;
  labels.assign(L, L + n);
  inst.assign(M, M + (size_t)n * nf);
  tsvm_free(L);
  tsvm_free(M);
  printf("Dataset size %ld #features %ld nnz=%ld sparsity=%3f%%\n", n, nf, (long)nnz,
         n && nf ? 100.0 * nnz / ((double)n * nf) : 0.0);
  return true;
}

// Decision values of the in-memory model on a test file, the accuracy line of the reference's
// (disabled) predict (tensorsvm-train.cu:223, 267).
bool run_test(tsvm_context *ctx, const Args &a, double gamma, const std::vector<float> &X,
              const std::vector<float> &y, const std::vector<double> &alpha, long n, long d,
              double b, int pos, int neg) {
  std::vector<float> tl, tx;
  long tn = 0, td = 0;
  printf("testfilepath=%s\n", a.test);
  if (!libsvm_read(a.test, a.scale256, tl, tx, tn, td)) return false;
  if (td != d) printf("training #feature(%ld) != testing feature (%ld)\n", d, td);
  const long dd = std::max(d, td);
  std::vector<float> T((size_t)tn * dd, 0.f);
  for (long i = 0; i < tn; ++i)
    for (long c = 0; c < td; ++c) T[(size_t)i * dd + c] = tx[(size_t)i * td + c];
  std::vector<float> sv;
  std::vector<double> coef;
  tsvm_model_view m{};
  m.d = (int32_t)dd;
  m.rho = -b;
  if (a.T == 0) {
    sv.assign(dd, 0.f);
    std::vector<double> w(d, 0.0);
    for (long j = 0; j < n; ++j)
      if (alpha[j] > 1e-6)
        for (long c = 0; c < d; ++c) w[c] += alpha[j] * y[j] * X[(size_t)j * d + c];
    for (long c = 0; c < d; ++c) sv[c] = (float)w[c];
    m.kernel = TSVM_KERNEL_LINEAR;
  } else {
    for (long j = 0; j < n; ++j)
      if (alpha[j] > 1e-6) {
        coef.push_back(y[j] * alpha[j]);
        for (long c = 0; c < dd; ++c) sv.push_back(c < d ? X[(size_t)j * d + c] : 0.f);
      }
    m.kernel = TSVM_KERNEL_RBF;
    m.nsv = (int64_t)coef.size();
    m.coef = coef.data();
    m.gamma = gamma;
  }
  m.sv = sv.data();
  std::vector<double> f(tn);
  const tsvm_status st = tsvm_predict(ctx, &m, T.data(), tn, f.data());
  if (st != TSVM_OK) {
    fprintf(stderr, "tensorsvm: %s\n", tsvm_status_string(st));
    return false;
  }
  long yes = 0;
  for (long i = 0; i < tn; ++i) {
    const double t = (int)tl[i] == pos ? 1.0 : (int)tl[i] == neg ? -1.0 : 0.0;
    if (f[i] * t > 0) ++yes;
  }
  printf("prediction accuracy %.3f (%ld/%ld)\n", tn ? 1.0 * yes / tn : 0.0, yes, tn);
  return true;
}

}  // namespace

int main(int argc, char **argv) {
  Args a;
  if (!parse(argc, argv, a)) {
    help_msg();
    return 1;
  }
  std::string model = a.model ? a.model : std::string(a.train) + ".model";
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<float> labels, X;
  long n = 0, d = 0;
  if (!libsvm_read(a.train, a.scale256, labels, X, n, d)) return 1;
  if (a.NN != 0 && a.NN < n) {
    printf("Truncating the input file to first %ld instances\n", a.NN);
    n = a.NN;
    labels.resize(n);
    X.resize((size_t)n * d);
  }
  // POS = first label, NEG = first different label (tensorsvm-train.cu:880-895)
  int pos = -42, neg = -42;
  for (long i = 0; i < n; ++i) {
    if (pos == -42) pos = (int)labels[i];
    else if (neg == -42 && pos != (int)labels[i]) {
      neg = (int)labels[i];
      break;
    }
  }
  if (neg == -42) {
    fprintf(stderr, "Error: training data has a single class\n");
    return 1;
  }
  for (long i = 0; i < n; ++i) {
    if ((int)labels[i] == pos) labels[i] = 1;
    else if ((int)labels[i] == neg) labels[i] = -1;
    else {
      fprintf(stderr, "Error: LABELS[%ld] %.3f\n", i, labels[i]);
      return 1;
    }
  }
  printf("found labels: %d(+1) %d(-1)\n", pos, neg);
  printf("Reading files took %.3f seconds\n",
         std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  if (a.S != 0) {
    printf("unimplemented pgd\n");
    return 1;
  }
  double gamma = a.g;
  if (a.T == 2 && !(gamma > 0)) gamma = 1.0 / (double)d;
  int precision = a.precision >= 0 ? a.precision : (a.tensorcore ? TSVM_PREC_FP16 : TSVM_PREC_FP32);
  if (precision != TSVM_PREC_FP32) printf("\033[31mUsing TensorCore \033[39m\n");

  tsvm_context *ctx = nullptr;
  tsvm_status st = tsvm_create(&ctx, 0);
  if (st != TSVM_OK) {
    fprintf(stderr, "tensorsvm: %s\n", tsvm_status_string(st));
    return 1;
  }
  tsvm_ipm_options opt;
  tsvm_ipm_default_options(&opt);
  opt.verbose = a.quiet ? 0 : 1;
  opt.rel_gap_tol = a.rel_gap;
  opt.max_iter = a.max_iter;
  opt.precision = precision == TSVM_PREC_FP32 ? TSVM_PREC_FP32 : TSVM_PREC_BF16;
  if (a.T == 0) printf("Linear SVM\n");
  else
    printf("\033[34mRBF kernel: gamma=%.3e, C=%.3e Approximation Rank K=%d\033[39m\n", gamma, a.C,
           a.K);
  std::vector<double> alpha(n);
  double b = 0;
  tsvm_factor_info finfo{};
  tsvm_ipm_stats istats{};
  const auto t1 = std::chrono::steady_clock::now();
  st = tsvm_train(ctx, X.data(), labels.data(), n, (int)d, a.T, gamma, a.C, a.K, precision, &opt,
                  alpha.data(), &b, &finfo, &istats);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
  if (st != TSVM_OK && st != TSVM_WARN_ILL_CONDITIONED && st != TSVM_WARN_MAX_ITER &&
      st != TSVM_ERR_NOT_SPD) {
    fprintf(stderr, "tensorsvm: %s\n", tsvm_status_string(st));
    tsvm_destroy(ctx);
    return 1;
  }
  if (a.T == 2) {
    printf("[LRA]: C: largest ew=%.3e, smallest ew=%.3e\n", finfo.eig_max, finfo.eig_min);
    printf("real rank is %d\n", finfo.realk);
    printf("\033[95mLRA elapsed time = %.4f seconds\033[39m\n", finfo.ms_total / 1e3);
  }
  printf("\033[95mMPC elapsed time = %.4f seconds\033[39m (%d iterations, %s)\n",
         istats.ms_total / 1e3, istats.iters, tsvm_status_string(st));
  printf("train elapsed time = %.4f seconds\n", secs);
  if (a.analysis && a.T == 2) {
    // ||K~||_F and ||K~ - Z Z^T||_F of this factor (the reference's -analysis, T:2328-2360)
    const auto ta = std::chrono::steady_clock::now();
    double kn = 0, kr = 0;
    st = tsvm_train_residual(ctx, &kn, &kr);
    if (st != TSVM_OK) {
      fprintf(stderr, "tensorsvm: %s\n", tsvm_status_string(st));
      tsvm_destroy(ctx);
      return 1;
    }
    printf("fnorm(K)=%.3e fnorm(K-U*U=%.3e')\n", kn, kr);
    printf("rbf_fnorm_res elapsed time = %.4f seconds\n",
           std::chrono::duration<double>(std::chrono::steady_clock::now() - ta).count());
  }
  printf("Writemodel ");
  const auto tw = std::chrono::steady_clock::now();
  int64_t nsv = 0, nfree = 0;
  st = tsvm_write_model(model.c_str(), a.T == 0 ? TSVM_KERNEL_LINEAR : TSVM_KERNEL_RBF, X.data(),
                        labels.data(), alpha.data(), n, (int32_t)d, a.C, gamma, b, pos, neg, 0,
                        &nsv, &nfree);
  printf("#BSV %lld, #SV %lld\n", (long long)nfree, (long long)nsv);
  if (st != TSVM_OK) fprintf(stderr, "Can't write %s\n", model.c_str());
  printf("elapsed time = %.4f seconds\n",
         std::chrono::duration<double>(std::chrono::steady_clock::now() - tw).count());
  printf("approx mean b=%.6e\n", b);
  bool ok = st == TSVM_OK;
  if (ok && a.test) ok = run_test(ctx, a, gamma, X, labels, alpha, n, d, b, pos, neg);
  tsvm_destroy(ctx);
  return ok ? 0 : 1;
}
