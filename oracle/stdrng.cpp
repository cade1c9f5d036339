// stdrng.cpp -- the C++ standard library's mt19937_64 and its uniform
// distributions behind a C interface, for the Connectome restatement in
// oracle/connectome.py.
//
// TEST INFRASTRUCTURE ONLY.  The reference draws its structural randomness
// from std::mt19937_64 through std::uniform_real_distribution<float> and
// std::uniform_int_distribution<int> (src/structure/connectome.cpp:49,66,
// 195-209); how a distribution maps engine output to values is left to the
// library, so the restatement calls the library (the same libstdc++ the
// reference is built with) instead of restating it.
#include <cstdint>
#include <random>

extern "C" {

void* srng_new(uint64_t seed) { return new std::mt19937_64(seed); }

void* srng_copy(void* h) { return new std::mt19937_64(*static_cast<std::mt19937_64*>(h)); }

void srng_free(void* h) { delete static_cast<std::mt19937_64*>(h); }

float srng_uniform_float(void* h, float a, float b) {
  std::uniform_real_distribution<float> d(a, b);
  return d(*static_cast<std::mt19937_64*>(h));
}

int srng_uniform_int(void* h, int a, int b) {
  std::uniform_int_distribution<int> d(a, b);
  return d(*static_cast<std::mt19937_64*>(h));
}

}  // extern "C"
