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
         "-prec fp32|bf16|fp16 : contraction precision (overrides -tensorcore)\n"
         "-rel_gap tol : also stop at relative duality gap <= tol\n"
         "-scale256 : divide feature values by 256\n"
         "-analysis : report ||K - Z Z'||_F / ||K||_F (not available in this build)\n"
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
                    : !strcmp(p, "fp16") ? TSVM_PREC_FP16 : -2;
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

// Two-pass LIBSVM reader with the reference's index rules: dense row-major float, indices
// shifted by the smallest index seen (1 for 1-based files), strictly increasing indices.
bool libsvm_read(const char *path, bool scale256, std::vector<float> &labels,
                 std::vector<float> &inst, long &n, long &nf) {
  FILE *f = fopen(path, "r");
  if (!f) {
    fprintf(stderr, "Can't open %s\n", path);
    return false;
  }
  std::vector<char> buf(1 << 20);
  std::vector<std::vector<std::pair<int, float>>> rows;
  long max_index = 0, min_index = 1, elements = 0, l = 0;
  std::string line;
  auto read_line = [&](std::string &out) -> bool {
    out.clear();
    while (fgets(buf.data(), (int)buf.size(), f)) {
      out.append(buf.data());
      if (!out.empty() && out.back() == '\n') return true;
    }
    return !out.empty();
  };
  while (read_line(line)) {
    ++l;
    char *s = &line[0];
    char *save = nullptr;
    char *label = strtok_r(s, " \t\n\r", &save);
    if (!label) {
      printf("Empty line at line %ld\n", l);
      fclose(f);
      return false;
    }
    char *end = nullptr;
    const double lab = strtod(label, &end);
    if (end == label || *end != '\0') {
      printf("Wrong input format at line %ld\n", l);
      fclose(f);
      return false;
    }
    std::vector<std::pair<int, float>> feats;
    int prev = -1;
    while (true) {
      char *idx = strtok_r(nullptr, ":", &save);
      char *val = strtok_r(nullptr, " \t\n\r", &save);
      if (!val) break;
      errno = 0;
      const long index = strtol(idx, &end, 10);
      if (end == idx || errno != 0 || *end != '\0' || index <= prev) {
        printf("Wrong input format at line %ld\n", l);
        fclose(f);
        return false;
      }
      prev = (int)index;
      errno = 0;
      float v = (float)strtod(val, &end);
      if (end == val || errno != 0 || (*end != '\0' && !isspace((unsigned char)*end))) {
        printf("Wrong input format at line %ld\n", l);
        fclose(f);
        return false;
      }
      if (scale256) v /= 256;
      feats.emplace_back((int)index, v);
      if (index < min_index) min_index = index;
      if (index > max_index) max_index = index;
      ++elements;
    }
    labels.push_back((float)lab);
    rows.push_back(std::move(feats));
  }
  fclose(f);
  n = (long)rows.size();
  nf = min_index == 0 ? max_index + 1 : max_index;
  inst.assign((size_t)n * nf, 0.f);
  for (long i = 0; i < n; ++i)
    for (auto &p : rows[i]) inst[(size_t)i * nf + (p.first - min_index)] = p.second;
  printf("Dataset size %ld #features %ld nnz=%ld sparsity=%3f%%\n", n, nf, elements,
         n && nf ? 100.0 * elements / ((double)n * nf) : 0.0);
  return true;
}

bool write_model(const char *path, const Args &a, double gamma, const std::vector<float> &X,
                 const std::vector<float> &y, const std::vector<double> &alpha, long n, long d,
                 double b, int pos, int neg) {
  std::vector<long> sv, freesv;
  for (long i = 0; i < n; ++i)
    if (alpha[i] > 1e-6) {
      sv.push_back(i);
      if (alpha[i] < a.C - 1e-6) freesv.push_back(i);
    }
  printf("#BSV %zu, #SV %zu\n", freesv.size(), sv.size());
  FILE *f = fopen(path, "w");
  if (!f) {
    fprintf(stderr, "Can't open %s\n", path);
    return false;
  }
  if (a.T == 0) {
    std::vector<double> w(d, 0.0);
    for (long j : sv)
      for (long c = 0; c < d; ++c) w[c] += alpha[j] * y[j] * X[(size_t)j * d + c];
    fprintf(f, "solver_type L2R_L1LOSS_SVC_DUAL\n");
    fprintf(f, "nr_class 2\n");
    fprintf(f, "label %d %d\n", pos, neg);
    fprintf(f, "nr_feature %ld\n", d);
    fprintf(f, "bias %d\n", 1);
    fprintf(f, "w\n");
    for (long c = 0; c < d; ++c) fprintf(f, "%.16f \n", w[c]);
    fprintf(f, "%.16f\n", b);
  } else {
    fprintf(f, "svm_type c_svc\n");
    fprintf(f, "kernel_type rbf\n");
    fprintf(f, "gamma %.7f\n", gamma);
    fprintf(f, "nr_class 2\n");
    fprintf(f, "total_sv %zu\n", sv.size());
    fprintf(f, "rho %f\n", -b);
    fprintf(f, "label %d %d\n", pos, neg);
    fprintf(f, "nr_sv %zu %zu\n", freesv.size(), sv.size() - freesv.size());
    fprintf(f, "SV\n");
    std::string line;
    char tmp[64];
    for (long j : sv) {
      line.clear();
      snprintf(tmp, sizeof tmp, "%7f ", y[j] * alpha[j]);
      line += tmp;
      for (long c = 0; c < d; ++c) {
        const float v = X[(size_t)j * d + c];
        if (v > 0 || v < 0) {
          snprintf(tmp, sizeof tmp, "%ld:%7f ", c + 1, v);
          line += tmp;
        }
      }
      line += '\n';
      fputs(line.c_str(), f);
    }
  }
  fclose(f);
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
  if (a.analysis) printf("-analysis is not available in this build; ignored\n");
  if (a.test) printf("-test not implemented\n");
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
  printf("Writemodel ");
  const bool ok = write_model(model.c_str(), a, gamma, X, labels, alpha, n, d, b, pos, neg);
  printf("approx mean b=%.6e\n", b);
  tsvm_destroy(ctx);
  return ok ? 0 : 1;
}
