// Drop-in for the reference header include/ftlm/lanczos_engine.hpp.
#pragma once

#include <complex>
#include <functional>
#include <utility>
#include <vector>

#include "ftlm/lanczos.hpp"

namespace ftlm {

/// Operator + three host buffers, with run_extrema = lanczos_extrema on the operator.
struct LanczosEngine {
  using ApplyH = std::function<void(const std::complex<double>*, std::complex<double>*)>;

  int dim = 0;
  ApplyH apply_h{};
  std::vector<std::complex<double>> v_cur{};
  std::vector<std::complex<double>> v_prev{};
  std::vector<std::complex<double>> work{};

  LanczosEngine() = default;
  LanczosEngine(int d, ApplyH fn) : dim(d), apply_h(std::move(fn)) { resize_buffers(d); }

  void resize_buffers(int d) {
    dim = d;
    v_cur.assign(static_cast<std::size_t>(d), std::complex<double>(0.0, 0.0));
    v_prev.assign(static_cast<std::size_t>(d), std::complex<double>(0.0, 0.0));
    work.assign(static_cast<std::size_t>(d), std::complex<double>(0.0, 0.0));
  }

  LanczosExtrema run_extrema(int max_steps, unsigned seed = 1) const {
    return lanczos_extrema(dim, apply_h, max_steps, seed);
  }
};

}  // namespace ftlm
