#pragma once
#include <functional>
#include <random>
#include <string>
#include <vector>

#include "common.hpp"

namespace gpuga {

struct Engine;

// Host GA (ga.cu).  `eval` scores the whole population at once: the engine's
// batched fitness, or a caller callback.
struct GA {
  GAParams gp;
  int d = 0;
  int child_number = 0;
  int generation = 0;
  std::vector<float> pmin, pmax, population, population_copy, fitness, cum;
  std::vector<int> index;
  std::mt19937 rng;
  std::function<int(int, const float*, float*)> eval;
  Engine* engine = nullptr;

  int init(int num_vars, const float* mn, const float* mx, const GAParams& params, unsigned seed);
  int step(std::string* line);
  void sort_population();
  std::string output_line() const;
  int get_a_parent();
  void crossover();
  void mutation();
};

}  // namespace gpuga
