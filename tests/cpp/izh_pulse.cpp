// Builds a small Izhikevich pulse network through the C++ mirror of the
// Network API (include/simuse_b200.hpp), runs it with an input current
// injected every step, and prints the per-step spike counts and the final v
// as text for the test that compares them with the Python mirror's run.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "simuse_b200.hpp"

int main(int argc, char **argv) {
  const uint32_t n = 400, k = 30, steps = argc > 1 ? (uint32_t)std::atoi(argv[1]) : 200;
  try {
    simuse::Network net(0);
    auto pop = net.add_population(simuse::Model::Izhikevich, n);
    const float params[7] = {0.5f, 0.02f, 0.2f, -65.0f, 8.0f, 0.0f, 30.0f};
    for (uint32_t c = 0; c < 7; ++c) net.fill_param(pop, c, params[c]);
    net.fill_state(pop, 0, -65.0f);
    net.fill_state(pop, 1, -13.0f);
    std::vector<uint32_t> pre, post;
    std::vector<float> w;
    std::vector<uint8_t> d;
    uint64_t h = 12345;
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t q = 0; q < k; ++q) {
        h = h * 6364136223846793005ull + 1442695040888963407ull;  // LCG, same as the test's twin
        pre.push_back(i);
        post.push_back((uint32_t)((h >> 33) % n));
        w.push_back(i < n * 4 / 5 ? 0.5f : -1.0f);
        d.push_back((uint8_t)(1 + (h >> 60) % 4));
      }
    net.connect(pop, pre, pop, post, w, d);
    net.build();
    std::vector<uint32_t> idx(n);
    std::vector<float> cur(n);
    for (uint32_t i = 0; i < n; ++i) {
      idx[i] = i;
      cur[i] = 4.0f + 0.02f * (float)(i % 50);
    }
    for (uint32_t t = 0; t < steps; ++t) {
      net.inject_current(pop, idx, cur);
      net.step(1);
      uint32_t c = 0;
      for (int32_t s : net.spikes(pop)) c += s != 0;
      std::printf("%u\n", c);
    }
    for (float v : net.state(pop, 0)) std::printf("%.9g\n", v);
    try {
      net.connect(pop, pre, pop, post, w, d);  // after build: the reference panics, here an exception
      return 3;
    } catch (const simuse::Error &e) {
      if (e.status() != SG_E_STATE) return 4;
    }
  } catch (const simuse::Error &e) {
    std::fprintf(stderr, "error %d: %s\n", e.status(), e.what());
    return 2;
  }
  return 0;
}
