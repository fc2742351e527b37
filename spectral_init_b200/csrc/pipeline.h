// spectral_init pipeline on the device.
#pragma once

#include <vector>

#include "solver.h"

namespace si {

struct PipelineConfig {
  int compute_mode = SI_COMPUTE_PYTHON_COMPAT;
  bool add_noise = true;
  SolverConfig solver;
};

struct PipelineReport {
  int n_components_graph = 0;
  SolverStats stats;
  std::vector<double> eigvals;
};

// graph and data device-resident; out_dev f32 [n x nc].
void spectral_init_pipeline(const Exec& ex, const GraphDev& g, int nc, uint64_t seed, const float* data_dev,
                            int64_t n_features, const PipelineConfig& pc, float* out_dev, PipelineReport& rep);

// embed_disconnected (src/multi_component.rs:16-74): f64 [n x nc] coordinates.
void embed_disconnected_dev(const Exec& ex, const GraphDev& g, const uint32_t* labels, int64_t ncomp, int nc,
                            uint64_t seed, const float* data_dev, int64_t n_features, const PipelineConfig& pc,
                            DevBuf<double>& result, PipelineReport& rep);

}  // namespace si
