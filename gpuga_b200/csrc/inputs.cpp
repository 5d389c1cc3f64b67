// Input formats of GPUGA: potential.in, train.in, ga.in.  Same read order,
// same FP32 storage and the same validation rules as the reference, with
// status codes in place of exit().
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "common.hpp"

namespace gpuga {

namespace {
thread_local std::string g_err;

struct FileCloser {
  void operator()(FILE* f) const {
    if (f) fclose(f);
  }
};
using FilePtr = std::unique_ptr<FILE, FileCloser>;

FilePtr open_in(const std::string& dir, const char* name) {
  std::string path = dir + "/" + name;
  FILE* f = fopen(path.c_str(), "r");
  if (!f) set_error("Failed to open %s.", path.c_str());
  return FilePtr(f);
}
}  // namespace

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

const char* last_error() { return g_err.c_str(); }

int cuda_status(cudaError_t e, const char* what, const char* file, int line) {
  set_error("CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
  cudaGetLastError();  // clear a sticky launch error so the caller can continue
  return (e == cudaErrorMemoryAllocation) ? GPUGA_ERR_OOM : GPUGA_ERR_CUDA;
}

int num_vars_for(int potential_type, int num_neurons) {
  switch (potential_type) {
    case 0: return 15;  // fitness.cu:237-240
    case 1: return 9;   // fitness.cu:241-244
    case 2: return 13;  // fitness.cu:245-248
    case 3: return num_neurons * (num_neurons + 4) + 1;  // fitness.cu:249-258
    case 4: return 15;  // RI parameters, anion charge -q
    default: return -1;
  }
}

// fitness.cu:220-314.  Keyword names are read and ignored; only order matters.
int read_potential_in(const std::string& dir, PotentialSpec* spec) {
  FilePtr f = open_in(dir, "potential.in");
  if (!f) return GPUGA_ERR_IO;
  char name[256];
  if (fscanf(f.get(), "%255s%d", name, &spec->type) != 2) {
    set_error("reading error for potential.in.");
    return GPUGA_ERR_PARSE;
  }
  if (spec->type == 3) {
    if (fscanf(f.get(), "%255s%d", name, &spec->num_neurons) != 2) {
      set_error("reading error for potential.in.");
      return GPUGA_ERR_PARSE;
    }
    if (spec->num_neurons < 1) {
      set_error("num_neurons should be positive.");
      return GPUGA_ERR_PARSE;
    }
  }
  spec->num_vars = num_vars_for(spec->type, spec->num_neurons);
  if (spec->num_vars < 0) {
    set_error("unsupported potential type.");
    return GPUGA_ERR_UNSUPPORTED;
  }
  spec->pmin.assign(spec->num_vars, 0.f);
  spec->pmax.assign(spec->num_vars, 0.f);
  if (fscanf(f.get(), "%255s%f", name, &spec->cutoff) != 2) {
    set_error("reading error for potential.in.");
    return GPUGA_ERR_PARSE;
  }
  float* w[3] = {&spec->w_force, &spec->w_energy, &spec->w_stress};
  const char* wname[3] = {"force", "energy", "stress"};
  for (int k = 0; k < 3; ++k) {
    if (fscanf(f.get(), "%255s%f", name, w[k]) != 2) {
      set_error("reading error for potential.in.");
      return GPUGA_ERR_PARSE;
    }
    if (*w[k] < 0) {
      set_error("weight for %s should >= 0", wname[k]);
      return GPUGA_ERR_PARSE;
    }
  }
  for (int n = 0; n < spec->num_vars; ++n) {
    if (spec->type != 3) {
      if (fscanf(f.get(), "%255s%f%f", name, &spec->pmin[n], &spec->pmax[n]) != 3) {
        set_error("reading error for potential.in.");
        return GPUGA_ERR_PARSE;
      }
    } else {  // fitness.cu:308-309
      spec->pmin[n] = -3.0f;
      spec->pmax[n] = 3.0f;
    }
  }
  return GPUGA_OK;
}

// fitness.cu:40-57 in FP32, operation order kept.  Compiled with
// -ffp-contract=off so the host compiler fuses nothing.
void box_inverse(float* h) {
  h[9] = h[4] * h[8] - h[5] * h[7];
  h[10] = h[2] * h[7] - h[1] * h[8];
  h[11] = h[1] * h[5] - h[2] * h[4];
  h[12] = h[5] * h[6] - h[3] * h[8];
  h[13] = h[0] * h[8] - h[2] * h[6];
  h[14] = h[2] * h[3] - h[0] * h[5];
  h[15] = h[3] * h[7] - h[4] * h[6];
  h[16] = h[1] * h[6] - h[0] * h[7];
  h[17] = h[0] * h[4] - h[1] * h[3];
  float volume = h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) +
                 h[2] * (h[3] * h[7] - h[4] * h[6]);
  for (int n = 9; n < 18; n++) h[n] /= volume;
}

// Validation of fitness.cu:163-218 and the FP64 normalisers of fitness.cu:86-160.
int finish_training_set(TrainingSet* ts) {
  if (ts->Nc < 2) {
    set_error("Number of configurations should >= 2");
    return GPUGA_ERR_PARSE;
  }
  if (ts->Nc_force < 1) {
    set_error("Number of force configurations should >= 1");
    return GPUGA_ERR_PARSE;
  }
  if (ts->Nc_force > ts->Nc - 1) {
    set_error("Number of potential configurations should >= 1");
    return GPUGA_ERR_PARSE;
  }
  ts->N = 0;
  ts->max_Na = 0;
  ts->Na_sum.assign(ts->Nc, 0);
  for (int c = 0; c < ts->Nc; ++c) {
    if (ts->Na[c] < 2) {
      set_error("Number of atoms %d should >= 2", ts->Na[c]);
      return GPUGA_ERR_PARSE;
    }
    if (c > 0) ts->Na_sum[c] = ts->Na_sum[c - 1] + ts->Na[c - 1];
    ts->N += ts->Na[c];
    if (ts->Na[c] > ts->max_Na) ts->max_Na = ts->Na[c];
  }
  ts->N_force = 0;
  for (int c = 0; c < ts->Nc_force; ++c) ts->N_force += ts->Na[c];
  const int N = ts->N, Nc = ts->Nc;
  double fss = 0, pss = 0, vss = 0;
  for (int i = 0; i < ts->N_force; ++i)
    for (int k = 0; k < 3; ++k) {
      double v = ts->force_ref[i + (size_t)N * k];
      fss += v * v;
    }
  float emin = 0.0f;  // fitness.cu:86, 103-104: E_min starts at 0
  for (int c = ts->Nc_force; c < Nc; ++c)
    if (ts->pe_ref[c] < emin) emin = ts->pe_ref[c];
  for (int c = ts->Nc_force; c < Nc; ++c) {
    double e = (double)ts->pe_ref[c] - (double)emin;
    pss += e * e;
    for (int k = 0; k < 6; ++k) {
      double v = ts->virial_ref[c + (size_t)Nc * k];
      vss += v * v;
    }
  }
  ts->norm_force = fss;
  ts->norm_energy = pss;
  ts->norm_virial = vss;
  return GPUGA_OK;
}

// fitness.cu:59-161 (read order, transposition of the box, FP32 storage).
int read_train_in(const std::string& dir, TrainingSet* ts) {
  FilePtr fp = open_in(dir, "train.in");
  if (!fp) return GPUGA_ERR_IO;
  FILE* f = fp.get();
  if (fscanf(f, "%d%d", &ts->Nc, &ts->Nc_force) != 2) {
    set_error("Reading error for train.in.");
    return GPUGA_ERR_PARSE;
  }
  if (ts->Nc < 2 || ts->Nc_force < 1 || ts->Nc_force > ts->Nc - 1) {
    ts->Na.assign(std::max(ts->Nc, 0), 2);
    return finish_training_set(ts);  // produces the reference's message
  }
  const int Nc = ts->Nc;
  ts->Na.assign(Nc, 0);
  long long Ntot = 0;
  for (int c = 0; c < Nc; ++c) {
    if (fscanf(f, "%d", &ts->Na[c]) != 1) {
      set_error("Reading error for train.in.");
      return GPUGA_ERR_PARSE;
    }
    if (ts->Na[c] < 2) {
      set_error("Number of atoms %d should >= 2", ts->Na[c]);
      return GPUGA_ERR_PARSE;
    }
    Ntot += ts->Na[c];
  }
  if (Ntot > (1LL << 30)) {
    set_error("train.in holds too many atoms (%lld).", Ntot);
    return GPUGA_ERR_UNSUPPORTED;
  }
  const int N = (int)Ntot;
  std::vector<int> Na_sum(Nc, 0);
  for (int c = 1; c < Nc; ++c) Na_sum[c] = Na_sum[c - 1] + ts->Na[c - 1];
  ts->type.assign(N, 0);
  ts->r.assign(3 * (size_t)N, 0.f);
  ts->h.assign(18 * (size_t)Nc, 0.f);
  ts->pe_ref.assign(Nc, 0.f);
  ts->virial_ref.assign(6 * (size_t)Nc, 0.f);
  ts->force_ref.assign(3 * (size_t)N, 0.f);
  float* v = ts->virial_ref.data();
  for (int c = 0; c < Nc; ++c) {
    if (c >= ts->Nc_force) {
      if (fscanf(f, "%f%f%f%f%f%f%f", &ts->pe_ref[c], &v[c], &v[c + Nc], &v[c + 2 * Nc], &v[c + 3 * Nc],
                 &v[c + 4 * Nc], &v[c + 5 * Nc]) != 7) {
        set_error("reading error for train.in.");
        return GPUGA_ERR_PARSE;
      }
    }
    float t[9];
    for (int k = 0; k < 9; ++k)
      if (fscanf(f, "%f", &t[k]) != 1) {
        set_error("reading error for train.in.");
        return GPUGA_ERR_PARSE;
      }
    float* h = ts->h.data() + 18 * (size_t)c;
    h[0] = t[0]; h[3] = t[1]; h[6] = t[2];
    h[1] = t[3]; h[4] = t[4]; h[7] = t[5];
    h[2] = t[6]; h[5] = t[7]; h[8] = t[8];
    box_inverse(h);
    for (int k = 0; k < ts->Na[c]; ++k) {
      const int i = Na_sum[c] + k;
      int cnt;
      if (c < ts->Nc_force) {
        cnt = fscanf(f, "%d%f%f%f%f%f%f", &ts->type[i], &ts->r[i], &ts->r[i + N], &ts->r[i + 2 * (size_t)N],
                     &ts->force_ref[i], &ts->force_ref[i + N], &ts->force_ref[i + 2 * (size_t)N]);
        if (cnt != 7) {
          set_error("reading error for train.in.");
          return GPUGA_ERR_PARSE;
        }
      } else {
        cnt = fscanf(f, "%d%f%f%f", &ts->type[i], &ts->r[i], &ts->r[i + N], &ts->r[i + 2 * (size_t)N]);
        if (cnt != 4) {
          set_error("reading error for train.in.");
          return GPUGA_ERR_PARSE;
        }
      }
    }
  }
  return finish_training_set(ts);
}

namespace {
// read_file.cu:46-72: splits one line into words, '#' starts a comment.
char* row_find_param(char* s, char* param[], int max_param, int* num_param) {
  *num_param = 0;
  int start_new_word = 1, comment_found = 0;
  if (s == NULL) return NULL;
  while (*s) {
    if (*s == '\n') {
      *s = '\0';
      return s + 1;
    } else if (comment_found) {
    } else if (*s == '#') {
      *s = '\0';
      comment_found = 1;
    } else if (isspace((unsigned char)*s)) {
      *s = '\0';
      start_new_word = 1;
    } else if (start_new_word) {
      if (*num_param < max_param) param[*num_param] = s;
      ++(*num_param);
      start_new_word = 0;
    }
    ++s;
  }
  return NULL;
}

// read_file.cu:74-101 (strtol base 0, strtod)
bool is_valid_int(const char* s, int* result) {
  if (s == NULL || *s == '\0') return false;
  char* p;
  errno = 0;
  *result = (int)strtol(s, &p, 0);
  return !(errno != 0 || s == p || *p != 0);
}

bool is_valid_real(const char* s, float* result) {
  if (s == NULL || *s == '\0') return false;
  char* p;
  errno = 0;
  *result = strtod(s, &p);
  return !(errno != 0 || s == p || *p != 0);
}
}  // namespace

// ga.cu:214-316
int read_ga_in(const std::string& dir, GAParams* ga) {
  std::string path = dir + "/ga.in";
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) {
    set_error("Failed to open %s.", path.c_str());
    return GPUGA_ERR_IO;
  }
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
  fclose(f);
  std::vector<char> content(text.begin(), text.end());
  content.push_back('\0');
  char* ptr = content.data();
  const int max_param = 10;
  char* param[max_param];
  int num_param;
  while (ptr) {
    ptr = row_find_param(ptr, param, max_param, &num_param);
    if (num_param == 0) continue;
    if (num_param > max_param) {
      set_error("too many words on one line of ga.in.");
      return GPUGA_ERR_PARSE;
    }
    if (strcmp(param[0], "maximum_generation") == 0) {
      if (num_param != 2) { set_error("maximum_generation should have 1 parameter."); return GPUGA_ERR_PARSE; }
      if (!is_valid_int(param[1], &ga->maximum_generation)) { set_error("maximum_generation should be integer."); return GPUGA_ERR_PARSE; }
      if (ga->maximum_generation < 1) { set_error("maximum_generation should be positive."); return GPUGA_ERR_PARSE; }
    } else if (strcmp(param[0], "population_size") == 0) {
      if (num_param != 2) { set_error("population_size should have 1 parameter."); return GPUGA_ERR_PARSE; }
      if (!is_valid_int(param[1], &ga->population_size)) { set_error("population_size should be integer."); return GPUGA_ERR_PARSE; }
      if (ga->population_size < 20) { set_error("population_size should >= 20."); return GPUGA_ERR_PARSE; }
      if (ga->population_size % 10 != 0) { set_error("population_size should be multiple of 10."); return GPUGA_ERR_PARSE; }
    } else if (strcmp(param[0], "parent_number") == 0) {
      if (num_param != 2) { set_error("parent_number should have 1 parameter."); return GPUGA_ERR_PARSE; }
      if (!is_valid_int(param[1], &ga->parent_number)) { set_error("parent_number should be integer."); return GPUGA_ERR_PARSE; }
      if (ga->parent_number < 10) { set_error("parent_number should >= 10."); return GPUGA_ERR_PARSE; }
      if (ga->parent_number % 10 != 0) { set_error("parent_number should be multiple of 10."); return GPUGA_ERR_PARSE; }
    } else if (strcmp(param[0], "mutation_rate") == 0) {
      if (num_param != 2) { set_error("mutation_rate should have 1 parameter."); return GPUGA_ERR_PARSE; }
      if (!is_valid_real(param[1], &ga->mutation_rate)) { set_error("mutation_rate should be a number."); return GPUGA_ERR_PARSE; }
      if (ga->mutation_rate < 0) { set_error("mutation_rate should >= 0."); return GPUGA_ERR_PARSE; }
      if (ga->mutation_rate > 1) { set_error("mutation_rate should <= 1."); return GPUGA_ERR_PARSE; }
    } else {
      set_error("'%s' is invalid keyword.", param[0]);
      return GPUGA_ERR_PARSE;
    }
  }
  return GPUGA_OK;
}

void decode_params(const PotentialSpec& spec, const float* x01, float* params) {
  for (int m = 0; m < spec.num_vars; ++m) {
    volatile float a = spec.pmin[m];
    volatile float b = spec.pmax[m] - a;
    volatile float bx = b * x01[m];
    params[m] = a + bx;
  }
}

}  // namespace gpuga
