// The reference's genetic algorithm (ga.cu:27-212), behaviour-identical:
// libstdc++ std::mt19937 with the same distribution objects drawn in the same
// order, FP32 cumulative selection probabilities, a stable ascending insertion
// sort, one-point crossover and a mutation count that decays linearly.
#include "ga.hpp"

#include <cmath>
#include <cstring>

namespace gpuga {

int GA::init(int num_vars, const float* mn, const float* mx, const GAParams& params, unsigned seed) {
  if (num_vars < 2) {
    set_error("the GA needs at least 2 variables (got %d).", num_vars);
    return GPUGA_ERR_ARG;
  }
  if (params.population_size < 2 || params.parent_number < 2 || params.parent_number > params.population_size ||
      (params.population_size - params.parent_number) % 2 != 0) {
    set_error("invalid GA sizes: population_size %d, parent_number %d.", params.population_size,
              params.parent_number);
    return GPUGA_ERR_ARG;
  }
  gp = params;
  d = num_vars;
  pmin.assign(mn, mn + d);
  pmax.assign(mx, mx + d);
  const int P = gp.population_size;
  child_number = P - gp.parent_number;  // ga.cu:32
  fitness.assign(P, 0.f);
  index.assign(P, 0);
  population.assign((size_t)P * d, 0.f);
  population_copy.assign((size_t)P * d, 0.f);
  cum.assign(gp.parent_number, 0.f);
  // ga.cu:41-46 (double intermediates stored to float, as written there)
  float numerator = 0.0;
  float denominator = (1.0 + gp.parent_number) * gp.parent_number / 2.0;
  for (int n = 0; n < gp.parent_number; ++n) {
    numerator += gp.parent_number - n;
    cum[n] = numerator / denominator;
  }
  rng = std::mt19937(seed);
  std::uniform_real_distribution<float> r1(0, 1);  // ga.cu:53-56
  for (int n = 0; n < P * d; ++n) population[n] = r1(rng);
  generation = 0;
  return GPUGA_OK;
}

// ga.cu:105-137
void GA::sort_population() {
  const int P = gp.population_size;
  for (int n = 0; n < P; ++n) index[n] = n;
  for (int i = 1; i < P; i++) {
    float key = fitness[i];
    int j = i - 1;
    while (j >= 0 && fitness[j] > key) {
      fitness[j + 1] = fitness[j];
      index[j + 1] = index[j];
      --j;
    }
    fitness[j + 1] = key;
    index[j + 1] = i;
  }
  population_copy = population;
  for (int n = 0; n < P; ++n)
    memcpy(&population[(size_t)n * d], &population_copy[(size_t)index[n] * d], sizeof(float) * d);
}

// ga.cu:138-147: "<generation> <best> <decoded elite...>" with %g
std::string ga_output_line(int generation, float best, const float* elite01, const float* pmin,
                           const float* pmax, int d) {
  std::string s;
  char buf[64];
  snprintf(buf, sizeof buf, "%d %g ", generation, best);
  s += buf;
  for (int m = 0; m < d; ++m) {
    volatile float a = pmin[m];
    volatile float b = pmax[m] - a;
    volatile float bx = b * elite01[m];
    float v = a + bx;
    snprintf(buf, sizeof buf, "%g ", v);
    s += buf;
  }
  s += "\n";
  return s;
}

std::string GA::output_line() const {
  return ga_output_line(generation, fitness[0], population.data(), pmin.data(), pmax.data(), d);
}

// ga.cu:200-212
int GA::get_a_parent() {
  int parent = 0;
  std::uniform_real_distribution<float> r1(0, 1);
  float reference_value = r1(rng);
  for (int n = 0; n < gp.parent_number; ++n) {
    if (cum[n] > reference_value) {
      parent = n;
      break;
    }
  }
  return parent;
}

int GA::mutation_count(int g) const {
  // ga.cu:190-192: rate in double stored to float, count rounded from float
  float rate_n = gp.mutation_rate * (1.0 - float(g) / gp.maximum_generation);
  int m = gp.population_size * d;
  return (int)std::round(m * rate_n);
}

// ga.cu:161-198, draws only.  Crossover (161-186): parents by rank, redrawn
// until they differ, point U{1, d-1}.  Mutation (188-198): the reference writes
// population[r1(rng)] = r2(rng) and is compiled as C++14, where GCC evaluates
// the index first; the order is explicit here.
void GA::draw_plan(int g, GenPlan* plan) {
  plan->pairs.resize((size_t)child_number / 2 * 3);
  for (int m = 0; m < child_number; m += 2) {
    int parent_1 = get_a_parent();
    int parent_2 = get_a_parent();
    while (parent_2 == parent_1) parent_2 = get_a_parent();
    std::uniform_int_distribution<int> r1(1, d - 1);
    int crossover_point = r1(rng);
    int* q = &plan->pairs[(size_t)m / 2 * 3];
    q[0] = parent_1;
    q[1] = parent_2;
    q[2] = crossover_point;
  }
  const int m = gp.population_size * d;
  const int count = mutation_count(g);
  std::vector<int> idx(count);
  std::vector<float> val(count);
  for (int n = 0; n < count; ++n) {
    std::uniform_int_distribution<int> r1(d, m - 1);
    std::uniform_real_distribution<float> r2(0, 1);
    idx[n] = r1(rng);
    val[n] = r2(rng);
  }
  // fold repeated genes: walking backwards, the first write seen is the one that stays
  if (stamp.size() != (size_t)m) stamp.assign(m, -1);
  ++stamp_tag;
  plan->mut_idx.clear();
  plan->mut_val.clear();
  for (int n = count - 1; n >= 0; --n) {
    if (stamp[idx[n]] == stamp_tag) continue;
    stamp[idx[n]] = stamp_tag;
    plan->mut_idx.push_back(idx[n]);
    plan->mut_val.push_back(val[n]);
  }
}

void GA::apply_plan(const GenPlan& plan) {
  for (int m = 0; m < child_number; m += 2) {
    const int* q = &plan.pairs[(size_t)m / 2 * 3];
    const int parent_1 = q[0], parent_2 = q[1], crossover_point = q[2];
    int child_1 = gp.parent_number + m;
    int child_2 = child_1 + 1;
    for (int n = 0; n < crossover_point; ++n) {
      population[(size_t)child_1 * d + n] = population[(size_t)parent_1 * d + n];
      population[(size_t)child_2 * d + n] = population[(size_t)parent_2 * d + n];
    }
    for (int n = crossover_point; n < d; ++n) {
      population[(size_t)child_1 * d + n] = population[(size_t)parent_2 * d + n];
      population[(size_t)child_2 * d + n] = population[(size_t)parent_1 * d + n];
    }
  }
  for (size_t n = 0; n < plan.mut_idx.size(); ++n) population[plan.mut_idx[n]] = plan.mut_val[n];
}

int GA::step(std::string* line) {
  const int P = gp.population_size;
  int s = eval(P, population.data(), fitness.data());
  if (s != GPUGA_OK) return s;
  sort_population();
  std::string l = output_line();
  if (line) *line = l;
  GenPlan plan;
  draw_plan(generation, &plan);
  apply_plan(plan);
  ++generation;
  return GPUGA_OK;
}

}  // namespace gpuga
