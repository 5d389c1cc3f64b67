#pragma once
#include <functional>
#include <random>
#include <string>
#include <vector>

#include "common.hpp"

namespace gpuga {

struct Engine;

// Everything a generation draws from the random stream (ga.cu:161-198).  The
// draws never depend on fitness values (parents are picked by rank from the
// fixed cumulative probabilities), so a generation's plan can be drawn before
// its population is scored, and the host and the device apply the same plan.
struct GenPlan {
  // per pair of children: parent_1, parent_2 (ranks < parent_number), crossover point
  std::vector<int> pairs;  // [child_number / 2][3]
  // mutations with later writes to the same gene already folded in (last one wins),
  // so they can be applied in any order: gene index into population[P*d], value
  std::vector<int> mut_idx;
  std::vector<float> mut_val;
};

// Host GA (ga.cu).  `eval` scores the whole population at once: the engine's
// batched fitness, or a caller callback.
struct GA {
  GAParams gp;
  int d = 0;
  int child_number = 0;
  int generation = 0;
  std::vector<float> pmin, pmax, population, population_copy, fitness, cum;
  std::vector<int> index;
  std::vector<int> stamp;  // per gene: last generation tag that wrote it while folding mutations
  int stamp_tag = 0;
  std::mt19937 rng;
  std::function<int(int, const float*, float*)> eval;
  Engine* engine = nullptr;

  int init(int num_vars, const float* mn, const float* mx, const GAParams& params, unsigned seed);
  int step(std::string* line);
  void sort_population();
  std::string output_line() const;
  int get_a_parent();
  // Draws generation `g`'s crossover and mutation choices in the reference's order.
  void draw_plan(int g, GenPlan* plan);
  // Crossover then mutation of the sorted population (ga.cu:161-198).
  void apply_plan(const GenPlan& plan);
  int mutation_count(int g) const;
};

// "<generation> <best> <decoded elite...>\n" with %g (ga.cu:138-147).
std::string ga_output_line(int generation, float best, const float* elite01, const float* pmin,
                           const float* pmax, int d);

}  // namespace gpuga
