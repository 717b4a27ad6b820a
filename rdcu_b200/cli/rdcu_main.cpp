// rdcu -- command-line front end of librdcu with the reference CLI's flags, input files
// and output files (reference rdcu.cu:599-1273 main and rdcu.cu:252-341 step_eval).
//
// usage: rdcu [-hvSFR] [-n NFIELDS] [-N NUMS] [-L LENGTHS] [-c COUPLING] [-A AMPLITUDE]
//             [-t TIME] [-d DT] [-s SEED] [-D DENSITY] [-g GPU] [-r RTOL] [-a ATOL] FILEBASE
//
// Parsing keeps the reference's semantics: getopt with GNU permutation, the last
// positional argument is FILEBASE and cancels -h, -N sets the dimension, -L values
// accumulate, -c/-coupling-file terms are "C,field,idx,pow,..." with the first value
// read as a double and the rest as integers, the amplitude defaults to 1e-3.  Where the
// reference overflows fixed buffers (100 ints per -c term, 2 values for -A, 1024
// characters per coupling-file token) this front end accepts the input instead.
#include <getopt.h>
#include <sys/time.h>
#include <unistd.h>

#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rdcu.h"

namespace {

// parse_list (rdcu.cu:343-357): integers separated by delim, at most max_len in total
void parse_int_list(const char* arg, std::vector<int>& lst, size_t max_len) {
  if (!arg) return;
  std::string copy(arg);
  char* save = nullptr;
  for (char* tok = strtok_r(&copy[0], ",", &save); tok; tok = strtok_r(nullptr, ",", &save)) {
    lst.push_back(atoi(tok));
    if (lst.size() >= max_len) return;
  }
}

// fparse_list (rdcu.cu:359-374): doubles into lst[*len..max_len), returns the characters
// consumed (strlen(token)+1 per token read)
int parse_double_list(const char* arg, double* lst, int* len, int max_len) {
  int chars = 0;
  if (!arg) return chars;
  std::string copy(arg);
  char* save = nullptr;
  for (char* tok = strtok_r(&copy[0], ",", &save); tok; tok = strtok_r(nullptr, ",", &save)) {
    chars += (int)strlen(tok) + 1;
    lst[(*len)++] = atof(tok);
    if (*len >= max_len) return chars;
  }
  return chars;
}

struct Term {
  double C;
  std::vector<int> ints;
};

// one coupling term (rdcu.cu:654-660, 831-834): one double, then integers from the
// character offset fparse_list reports
bool parse_term(const char* arg, std::vector<Term>& terms) {
  double C = 0;
  int one = 0;
  const int chars = parse_double_list(arg, &C, &one, 1);
  if (one == 0) return false;
  Term t;
  t.C = C;
  const size_t len = strlen(arg);
  if ((size_t)chars <= len) parse_int_list(arg + chars, t.ints, 1024);
  terms.push_back(t);
  return true;
}

double elapsed_since(const timeval& start) {
  timeval end;
  gettimeofday(&end, nullptr);
  return end.tv_sec - start.tv_sec + 1e-6 * (end.tv_usec - start.tv_usec);
}

// Output files written behind the integration: one background thread runs the writes in
// the order they were issued, from host copies of the state taken when the library
// delivers them, so the GPU keeps stepping while states.dat, times.dat and fs.dat are
// written.  Host buffers are recycled (at most kBuffers in flight; a new output waits for
// a free one), and drain() waits for every write -- the contents and order of each file
// are those of synchronous writes.
class Writer {
 public:
  static constexpr int kBuffers = 3;
  Writer() {
    for (int i = 0; i < kBuffers; ++i) free_.push_back(std::make_unique<std::vector<double>>());
    th_ = std::thread([this] { run(); });
  }
  ~Writer() {
    drain();
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_.notify_all();
    th_.join();
  }
  // a buffer for the next output (waits while all are queued for writing)
  std::unique_ptr<std::vector<double>> acquire() {
    std::unique_lock<std::mutex> g(m_);
    cv_.wait(g, [this] { return !free_.empty(); });
    auto b = std::move(free_.back());
    free_.pop_back();
    return b;
  }
  // runs task(buffer) on the writer thread, then recycles the buffer
  void submit(std::unique_ptr<std::vector<double>> b, std::function<void(const std::vector<double>&)> task) {
    {
      std::lock_guard<std::mutex> g(m_);
      q_.emplace_back(std::move(b), std::move(task));
    }
    cv_.notify_all();
  }
  void drain() {
    std::unique_lock<std::mutex> g(m_);
    cv_.wait(g, [this] { return q_.empty() && !busy_; });
  }

 private:
  using Job = std::pair<std::unique_ptr<std::vector<double>>, std::function<void(const std::vector<double>&)>>;
  std::mutex m_;
  std::condition_variable cv_;
  std::deque<Job> q_;
  std::vector<std::unique_ptr<std::vector<double>>> free_;
  bool stop_ = false, busy_ = false;
  std::thread th_;

  void run() {
    std::unique_lock<std::mutex> g(m_);
    for (;;) {
      cv_.wait(g, [this] { return stop_ || !q_.empty(); });
      if (q_.empty()) return;
      Job j = std::move(q_.front());
      q_.pop_front();
      busy_ = true;
      g.unlock();
      j.second(*j.first);
      g.lock();
      free_.push_back(std::move(j.first));
      busy_ = false;
      cv_.notify_all();
    }
  }
};

struct Ctx {
  rdcu_t* h = nullptr;
  int n = 1, ndim = 1, dense = 1, stiff = 0, verbose = 0;
  long long N = 0, nN = 0, nY = 0;
  double t0 = 0, t1 = 0;
  int steps = 0;
  timeval start{};
  std::string filebase;
  FILE *out = nullptr, *outsteps = nullptr, *outtimes = nullptr, *outstates = nullptr, *outf = nullptr,
       *outY = nullptr, *outrows = nullptr, *outcols = nullptr, *outvals = nullptr;
  std::vector<double> yloc, floc, Yloc, valsloc;
  std::vector<int> rowsloc, colsloc;
  long long nnz_max = 0;
  int failed = 0;
  Writer* writer = nullptr;
};

int check(Ctx& c, int rc, const char* what) {
  if (rc != RDCU_OK) {
    fprintf(stderr, "%s failed: %s (%s)\n", what, rdcu_error_string(rc), rdcu_last_error(c.h));
    if (c.out) fprintf(c.out, "%s failed: %s (%s)\n", what, rdcu_error_string(rc), rdcu_last_error(c.h));
    c.failed = rc;
  }
  return rc;
}

// f, Y and Jacobian dumps of one state (rdcu.cu:281-304, 1164-1190)
int write_derived(Ctx& c, const double* y, double t) {
  if (c.dense >= 2) {
    if (check(c, rdcu_rhs(c.h, t, y, c.floc.data(), c.dense >= 3 ? c.Yloc.data() : nullptr), "rhs")) return 1;
    fwrite(c.floc.data(), sizeof(double), c.nN, c.outf);
    fflush(c.outf);
    if (c.dense >= 3) {
      fwrite(c.Yloc.data(), 2 * sizeof(double), c.nN * c.nY, c.outY);
      fflush(c.outY);
    }
  }
  return 0;
}

int write_jac(Ctx& c, const double* y, double t) {
  int nnz = 0;
  if (check(c, rdcu_jac(c.h, t, y, &nnz, c.rowsloc.data(), c.colsloc.data(), c.valsloc.data()), "jac")) return 1;
  fwrite(c.rowsloc.data(), sizeof(int), c.nN + 1, c.outrows);
  fwrite(c.colsloc.data(), sizeof(int), nnz, c.outcols);
  fwrite(c.valsloc.data(), sizeof(double), nnz, c.outvals);
  fflush(c.outrows);
  fflush(c.outcols);
  fflush(c.outvals);
  return 0;
}

// step_eval (rdcu.cu:252-341), driven by the library's events
int on_event(void* user, const rdcu_event* ev) {
  Ctx& c = *static_cast<Ctx*>(user);
  if (ev->kind == RDCU_EV_ATTEMPT) {
    if (c.dense >= 1) {
      const double hh = ev->h;
      fwrite(&hh, sizeof(double), 1, c.outsteps);
    }
    if (ev->accepted) c.steps++;
    return 0;
  }
  if (ev->kind == RDCU_EV_EVAL) {
    if (c.dense >= 1) {
      auto b = c.writer->acquire();
      b->resize((size_t)c.nN);
      if (check(c, rdcu_memcpy(c.h, b->data(), ev->y, (unsigned long long)c.nN * sizeof(double)), "copy")) {
        c.writer->submit(std::move(b), [](const std::vector<double>&) {});
        return 1;
      }
      const double te = ev->t_eval;
      FILE *fst = c.outstates, *ftm = c.outtimes;
      c.writer->submit(std::move(b), [fst, ftm, te](const std::vector<double>& y) {
        fwrite(y.data(), sizeof(double), y.size(), fst);
        fflush(fst);
        fwrite(&te, sizeof(double), 1, ftm);
        fflush(ftm);
      });
    }
    if (write_derived(c, ev->y, ev->t_eval)) return 1;
    if (c.dense >= 4 && write_jac(c, ev->y, ev->t_eval)) return 1;
    return 0;
  }
  // checkpoint: progress line and fs.dat
  const double t = ev->t, h = ev->h;
  const double el = elapsed_since(c.start);
  const double frac = (t - c.t0) / (c.t1 - c.t0);
  const double eta = el / ((t - c.t0 + h) / (c.t1 - c.t0)) * (1 - frac);
  if (c.verbose) {
    printf("%.3f\t%1.3e\t%1.3e\t%f\t%i\t\r", frac, el, eta, h, c.steps);
    fflush(stdout);
  }
  fprintf(c.out, "%.3f\t%1.3e\t%1.3e\t%f\t%i\t\n", frac, el, eta, h, c.steps);
  fflush(c.out);
  const std::string file = c.filebase + "fs.dat";
  const int order = ev->order;
  const long long nblk = c.stiff ? 1 + order : 1;
  auto b = c.writer->acquire();
  b->resize((size_t)(c.nN * nblk));
  if (check(c, rdcu_memcpy(c.h, b->data(), ev->y, (unsigned long long)(c.nN * nblk) * sizeof(double)), "copy")) {
    c.writer->submit(std::move(b), [](const std::vector<double>&) {});
    return 1;
  }
  const long long nN = c.nN;
  const int stiff = c.stiff;
  c.writer->submit(std::move(b), [file, nN, t, h, stiff, order](const std::vector<double>& buf) {
    FILE* fs = fopen(file.c_str(), "wb");
    if (!fs) return;
    fwrite(buf.data(), sizeof(double), nN, fs);
    fwrite(&t, sizeof(double), 1, fs);
    fwrite(&h, sizeof(double), 1, fs);
    if (stiff) {
      fwrite(&order, sizeof(int), 1, fs);
      for (int i = 1; i <= order; i++) fwrite(buf.data() + (size_t)nN * i, sizeof(double), nN, fs);
    }
    fflush(fs);
    fclose(fs);
  });
  return 0;
}

void print_help(int n, int ndim) {
  printf("usage:\trdcu [-hvSFR] [-n NFIELDS] [-N NUMS] [-L LENGTHS]\n");
  printf("\t[-c COUPLING] [-A AMPLITUDE] [-t TIME] [-d DT] [-s SEED] \n");
  printf("\t[-D DENSITY] [-g GPU] [-r RTOL] [-a ATOL]  FILEBASE \n\n");
  printf("-h for help. Call with -n and -N to see Y indices. \n");
  printf("-v for verbose output, including progress \n");
  printf("-S for stiff system. Use the BDF method with finite differences instead of RK45 pseudospectral method. \n");
  printf("-F for fixed timestep \n");
  printf("-R to reload final state from FILEBASEfs.dat if possible\n");
  printf("NFIELDS is the number of fields. Default 1\n");
  printf("NUMS is number of grid points in each dimension (up to three), separated by commas (no spaces). Default 128\n");
  printf("LENGTHS is domain length in each dimension (up to three), separated by commas (no spaces). Default 1.0\n");
  printf("COUPLING is a list of coupling terms, separated by commas (no spaces). Default empty\n");
  printf("\tThe first value is the term coefficent. \n");
  printf("\tThe second value is an integer specifying the field that the term appears in. \n");
  printf("\tThe following 2N values are pairs of integers specifing the indices and powers for each factor that appear in the term. \n");
  printf("\tFactor indices for the given -n and -N values appear below. \n");
  printf("\tYou may specify additional coupling terms on separate lines in this format in the input file FILEBASEcoupling.dat. \n");
  printf("AMPLITUDE is uniform random initial condition amplitude. Default 1.0 \n");
  printf("\tYou may also provide a binary input file FILEBASEic.dat with the initial condition\n");
  printf("TIME is total integration time. Default 1e2 \n");
  printf("DT is the time between outputs. Default 1e0 \n");
  printf("\t You may include firststep, minstep, maxstep as additional comma-separated values \n");
  printf("\t If not included, the first step is 1/100th the value of dt \n");
  printf("SEED is random seed. Default 1 \n");
  printf("GPU is the index of the gpu. Default 0\n");
  printf("DENSITY is the output density. Default 1\n");
  printf("\t1 for the timesteps (FILEBASEtimes.dat) and evaluated state values (FILEBASEstates.dat), \n");
  printf("\t2 to include time derivatives (FILEBASEf.dat), 3 to include factors (FILEBASEY.dat), \n");
  printf("\t4 to include CSR Jacobian elements (FILEBASErows.dat, FILEBASEcols.dat, and FILEBASEvals.dat). \n");
  printf("RTOL is relative error tolerance. Default 1E-8\n");
  printf("ATOL is absolute error tolerance. Default 1E-8\n");
  printf("FILEBASE is base file name for output. \n");
  printf("\n");
  printf("Example: ./rdcu -N 128,128 -L 100.0,100.0 -n 2 -c 1.0,0,0,1 -c 1.0,0,6,1 -c 1.0,0,12,1 -c -2.0,0,7,1 -c -2.0,0,13,1 -c -1.0,0,0,3 -c -1.0,0,0,1,1,2 -c -0.8,0,0,2,1,1 -c -0.8,0,1,3 -c 1.0,1,1,1 -c 1.0,1,7,1 -c 1.0,1,13,1 -c 2.0,1,6,1 -c 2.0,1,12,1 -c -1.0,1,0,2,1,1 -c -1.0,1,1,3 -c 0.8,1,0,3 -c 0.8,1,0,1,1,2 -v -D3 2dcgle\n");
  printf("\n");
  printf("Indices for %i field(s) in %i dimension(s):\n", n, ndim);
  int l = 0;
  for (int i = 0; i < n; i++) printf("%i: u%i\n", l++, i);
  for (int j = 0; j < ndim; j++)
    for (int i = 0; i < n; i++) printf("%i: u%i_%i\n", l++, i, j);
  for (int j = 0; j < ndim; j++)
    for (int k = 0; k < ndim; k++)
      for (int i = 0; i < n; i++) printf("%i: u%i_%i%i\n", l++, i, j, k);
}

}  // namespace

int main(int argc, char* argv[]) {
  Ctx c;
  gettimeofday(&c.start, nullptr);

  double t1 = 1e2, dt = 1e0, atl = 1e-8, rtl = 1e-8, A = 1E-3, A0 = 0.0;
  double h = 0.0, hmin = 0, hmax = INFINITY;
  int gpu = 0, seed = 1, fixed = 0, n = 1, ndim = 1, ndim2 = 0, verbose = 0, help = 1, dense = 1, stiff = 0,
      reload = 0;
  int Nsloc[3] = {128, 128, 128};
  double Lsloc[3] = {1.0, 1.0, 1.0};
  std::vector<Term> terms;
  const char* filebase = nullptr;
  int ch;
  while (optind < argc) {
    if ((ch = getopt(argc, argv, "hvFRSn:N:L:c:A:t:d:s:D:g:r:a:")) != -1) {
      switch (ch) {
        case 'h': help = 1; break;
        case 'v': verbose = 1; break;
        case 'F': fixed = 1; break;
        case 'R': reload = 1; break;
        case 'S': stiff = 1; break;
        case 'n': if (optarg) n = atoi(optarg); break;
        case 'N':
          if (optarg) {
            std::vector<int> v;
            parse_int_list(optarg, v, 3);
            ndim = (int)v.size();
            for (int i = 0; i < ndim; ++i) Nsloc[i] = v[i];
          }
          break;
        case 'L':
          if (optarg && ndim2 < 3) parse_double_list(optarg, Lsloc, &ndim2, 3);
          break;
        case 'c':
          if (optarg) parse_term(optarg, terms);
          break;
        case 'A':
          if (optarg) {
            double As[4];
            int nAs = 0;
            parse_double_list(optarg, As, &nAs, 4);
            A = As[0];
            if (nAs > 1) A0 = As[1];
          }
          break;
        case 't': if (optarg) t1 = atof(optarg); break;
        case 'd':
          if (optarg) {
            double dts[4];
            int ndts = 0;
            parse_double_list(optarg, dts, &ndts, 4);
            dt = dts[0];
            if (ndts > 1) h = dts[1];
            if (ndts > 2) hmin = dts[2];
            if (ndts > 3) hmax = dts[3];
          }
          break;
        case 's': if (optarg) seed = atoi(optarg); break;
        case 'D': if (optarg) dense = atoi(optarg); break;
        case 'g': if (optarg) gpu = atoi(optarg); break;
        case 'r': if (optarg) rtl = atof(optarg); break;
        case 'a': if (optarg) atl = atof(optarg); break;
        default: break;
      }
    } else {
      filebase = argv[optind];
      optind++;
      help = 0;
    }
  }

  if (help) {
    print_help(n, ndim);
    return 0;
  }

  std::vector<std::string> sterms;
  for (int i = 0; i < n; i++) sterms.push_back("u" + std::to_string(i));
  for (int j = 0; j < ndim; j++)
    for (int i = 0; i < n; i++) sterms.push_back("u" + std::to_string(i) + "_" + std::to_string(j));
  for (int j = 0; j < ndim; j++)
    for (int k = 0; k < ndim; k++)
      for (int i = 0; i < n; i++)
        sterms.push_back("u" + std::to_string(i) + "_" + std::to_string(j) + std::to_string(k));

  if (ndim2 < ndim)
    printf("Warning: Number of length scales %i smaller than number of dimensions %i. Using defaults.\n", ndim2, ndim);

  c.filebase = filebase;
  std::string file = c.filebase + ".out";
  c.out = fopen(file.c_str(), "w");
  if (!c.out) {
    fprintf(stderr, "cannot open %s\n", file.c_str());
    return EXIT_FAILURE;
  }
  for (int i = 0; i < argc; i++) fprintf(c.out, "%s ", argv[i]);
  fprintf(c.out, "\n");
  fflush(c.out);

  file = c.filebase + "coupling.dat";
  if (FILE* in = fopen(file.c_str(), "r")) {
    if (verbose) {
      printf("Using coupling terms from file\n");
      fprintf(c.out, "Using coupling terms from file\n");
    }
    char* tok = nullptr;
    while (fscanf(in, "%ms", &tok) == 1) {
      parse_term(tok, terms);
      free(tok);
      tok = nullptr;
    }
    fclose(in);
  }

  const int nY = 1 + ndim + ndim * ndim;
  auto sterm = [&](int k) -> std::string {
    return (k >= 0 && k < (int)sterms.size()) ? sterms[k] : std::string("?");
  };
  if (verbose) {
    for (int k = 0; k < n; k++) {
      printf("%s'=", sterm(k).c_str());
      fprintf(c.out, "%s'=", sterm(k).c_str());
      for (auto& t : terms) {
        const int field = t.ints.empty() ? 0 : t.ints[0];
        if (field != k) continue;
        printf("%.3f", t.C);
        fprintf(c.out, "%.3f", t.C);
        const int np = (int)t.ints.size();
        for (int j = 1; j < np; j += 2) {
          const int pw = j + 1 < np ? t.ints[j + 1] : 0;
          printf("(%s)^%i", sterm(t.ints[j]).c_str(), pw);
          fprintf(c.out, "(%s)^%i", sterm(t.ints[j]).c_str(), pw);
        }
        printf(" + ");
        fprintf(c.out, " + ");
      }
      printf("0\n");
      fprintf(c.out, "0\n");
    }
  }
  fflush(stdout);
  fflush(c.out);

  double t = 0;
  long long N = Nsloc[0];
  for (int i = 1; i < ndim; i++) N *= Nsloc[i];
  const long long nN = N * n;
  c.n = n;
  c.ndim = ndim;
  c.N = N;
  c.nN = nN;
  c.nY = nY;
  c.dense = dense;
  c.stiff = stiff;
  c.verbose = verbose;
  c.yloc.assign((size_t)nN * 8, 0.0);

  if (h <= 0.0) h = fixed ? dt : dt / 100;

  // initial conditions (rdcu.cu:926-1008)
  file = c.filebase + "ic.dat";
  int loaded = 0, order = 0;
  if (FILE* in = fopen(file.c_str(), "r")) {
    loaded = 1;
    printf("Using initial conditions from file\n");
    fprintf(c.out, "Using initial conditions from file\n");
    size_t rd = fread(c.yloc.data(), sizeof(double), nN, in);
    if ((long long)rd != nN) {
      loaded = 0;
      printf("initial conditions file not compatible with N!\n");
      fprintf(c.out, "initial conditions file not compatible with N!\n");
    }
    fclose(in);
  }
  file = c.filebase + "fs.dat";
  int reloaded = 0;
  FILE* in = nullptr;
  if (reload && (in = fopen(file.c_str(), "r"))) {
    reloaded = 1;
    loaded = 1;
    printf("Reloading final conditions from file\n");
    fprintf(c.out, "Reloading final conditions from file\n");
    size_t rd = fread(c.yloc.data(), sizeof(double), nN, in);
    if ((long long)rd != nN) {
      printf("final conditions file not compatible with N!\n");
      fprintf(c.out, "final conditions file not compatible with N!\n");
      reloaded = 0;
      loaded = 0;
    }
    if (reloaded) {
      rd = fread(&t, sizeof(double), 1, in);
      rd = fread(&h, sizeof(double), 1, in);
      if (rd != 1) {
        printf("Couldn't read start time and step!\n");
        fprintf(c.out, "Couldn't read start time and step!\n");
        reloaded = 0;
      }
      if (stiff) {
        rd = fread(&order, sizeof(int), 1, in);
        if (rd != 1) {
          printf("Couldn't read order!\n");
          fprintf(c.out, "Couldn't read order!\n");
          order = 0;
          reloaded = 0;
        } else if (order < 0 || order > 7) {
          printf("Couldn't read order!\n");
          fprintf(c.out, "Couldn't read order!\n");
          order = 0;
          reloaded = 0;
        } else {
          rd = fread(c.yloc.data() + nN, sizeof(double), (size_t)nN * order, in);
          if ((long long)rd != nN * order) {
            printf("Couldn't read backwards differences!\n");
            fprintf(c.out, "Couldn't backwards differences!\n");
            reloaded = 0;
          }
        }
      }
    }
    fclose(in);
    printf("Restarting at t=%f with h=%f\n", t, h);
    fprintf(c.out, "Restarting at t=%f with h=%f\n", t, h);
  }
  if (!reloaded && !loaded) {
    printf("Using random initial conditions\n");
    fprintf(c.out, "Using random initial conditions\n");
    rdcu_random_ic(c.yloc.data(), n, N, A, A0, seed);
    FILE* fs = fopen(file.c_str(), "wb");
    if (fs) {
      fwrite(c.yloc.data(), sizeof(double), nN, fs);
      fwrite(&t, sizeof(double), 1, fs);
      fwrite(&h, sizeof(double), 1, fs);
      fclose(fs);
    }
  }
  fflush(c.out);
  fflush(stdout);

  const char* wt = loaded ? "ab" : "wb";
  auto open_out = [&](const char* suffix) { return fopen((c.filebase + suffix).c_str(), wt); };
  if (dense >= 1) {
    c.outsteps = open_out("steps.dat");
    c.outtimes = open_out("times.dat");
    c.outstates = open_out("states.dat");
  }
  if (dense >= 2) c.outf = open_out("f.dat");
  if (dense >= 3) c.outY = open_out("Y.dat");
  if (dense >= 4) {
    c.outrows = open_out("rows.dat");
    c.outcols = open_out("cols.dat");
    c.outvals = open_out("vals.dat");
  }

  // output times (rdcu.cu:1052-1059)
  const int n0 = int(t / dt) + 1;
  const int n1 = int(t1 / dt) + 1;
  std::vector<double> t_eval;
  for (int nn = n0; nn < n1; nn++) t_eval.push_back(dt * nn);

  // the library handle (problem set-up of rdcu.cu:863-1153)
  std::vector<double> Cs;
  std::vector<int> nprods;
  std::vector<const int*> cptr;
  for (auto& tm : terms) {
    Cs.push_back(tm.C);
    nprods.push_back((int)tm.ints.size());
    cptr.push_back(tm.ints.data());
  }
  rdcu_spec spec{};
  spec.n = n;
  spec.ndim = ndim;
  for (int a = 0; a < 3; ++a) {
    spec.Ns[a] = a < ndim ? Nsloc[a] : 1;
    spec.Ls[a] = a < ndim ? Lsloc[a] : 1.0;
  }
  spec.nterms = (int)terms.size();
  spec.C = Cs.data();
  spec.nprods = nprods.data();
  spec.c = cptr.data();
  spec.method = stiff ? RDCU_METHOD_BDF : RDCU_METHOD_DP45;
  spec.fixed = fixed;
  spec.rtol = rtl;
  spec.atol = atl;
  spec.device = gpu;
  int rc = rdcu_create(&c.h, &spec);
  if (rc != RDCU_OK) {
    printf("rdcu initialization failed: %s\n", rdcu_last_error(nullptr));
    fprintf(c.out, "rdcu initialization failed: %s\n", rdcu_last_error(nullptr));
    fclose(c.out);
    return EXIT_FAILURE;
  }
  rdcu_info info{};
  rdcu_get_info(c.h, &info);
  c.nnz_max = info.nnz_max;
  c.floc.assign((size_t)nN, 0.0);
  if (dense >= 3) c.Yloc.assign((size_t)nN * nY * 2, 0.0);
  if (dense >= 4) {
    c.rowsloc.assign((size_t)nN + 1, 0);
    c.colsloc.assign((size_t)std::max<long long>(1, c.nnz_max), 0);
    c.valsloc.assign((size_t)std::max<long long>(1, c.nnz_max), 0.0);
  }
  c.t0 = t;
  c.t1 = t1;
  if (check(c, rdcu_set_state(c.h, t, h, c.yloc.data(), stiff ? order : 0, stiff && order > 0 ? c.yloc.data() + nN : nullptr),
            "set_state"))
    return EXIT_FAILURE;

  // initial outputs (rdcu.cu:1155-1191)
  if (dense >= 1 && !reload) {
    fwrite(c.yloc.data(), sizeof(double), nN, c.outstates);
    fflush(c.outstates);
    fwrite(&t, sizeof(double), 1, c.outtimes);
    fflush(c.outtimes);
  }
  if (dense >= 2 && !reload) {
    if (write_derived(c, c.yloc.data(), t)) return EXIT_FAILURE;
    if (dense >= 4 && stiff && write_jac(c, c.yloc.data(), t)) return EXIT_FAILURE;
  }

  {
    Writer writer;
    c.writer = &writer;
    rc = rdcu_solve(c.h, t1, hmin, hmax, t_eval.data(), (int)t_eval.size(), on_event, &c);
    if (rc != RDCU_OK && rc != RDCU_ERR_CALLBACK) check(c, rc, "solve");
    writer.drain();
    c.writer = nullptr;
  }

  const double runtime = elapsed_since(c.start);
  printf("\nruntime: %f\n", runtime);
  fprintf(c.out, "\nsteps: %i\n", c.steps);
  fprintf(c.out, "runtime: %f\n", runtime);
  fflush(c.out);
  fclose(c.out);
  FILE* files[] = {c.outtimes, c.outsteps, c.outstates, c.outf, c.outY, c.outrows, c.outcols, c.outvals};
  for (FILE* f : files)
    if (f) fclose(f);
  rdcu_destroy(c.h);
  return (c.failed && c.failed != RDCU_ERR_CALLBACK) ? EXIT_FAILURE : 0;
}
