// Host-side BSIM4 set-up: model-card processing and the temperature / geometry precompute that
// turns (model card, instance parameters, temperature) into the per-record constant table the
// load kernel reads. This is set-up work, done once per circuit (or per temperature change).
#pragma once

#include <string>
#include <utility>
#include <vector>

namespace xb4 {

struct ModelSpec {
  bool pmos = false;
  std::vector<std::pair<std::string, double>> params;  // netlist name (any case) -> value
};

struct SetupOptions {
  double temp_c = 27.0;  // circuit temperature (.OPTIONS DEVICE TEMP), Celsius
  double tnom_c = 27.0;  // default nominal temperature (.OPTIONS DEVICE TNOM), Celsius
};

struct RecordTable {
  int n_records = 0;
  std::vector<double> tab;     // field-major: tab[f * n_records + r]
  std::vector<int> inst_rec;   // record index of each instance
};

// Builds the record table for n_inst BSIM4 instances.
//   inst_model[i]                 model index of instance i
//   inst_param_names              instance parameter names (L, W, NF, AD, AS, PD, PS, NRD, NRS,
//                                 SA, SB, SD, DELVTO, M, TEMP, ...)
//   inst_param_values[i*np + k]   value of parameter k for instance i; NaN = not given
// Returns an empty string on success, otherwise a description of the first unsupported or
// invalid input.
std::string build_records(const std::vector<ModelSpec> &models, int n_inst, const int *inst_model,
                          const std::vector<std::string> &inst_param_names,
                          const double *inst_param_values, const SetupOptions &opts, RecordTable &out);

}  // namespace xb4
