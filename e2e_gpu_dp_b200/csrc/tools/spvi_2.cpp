// Drop-in replacement for the reference's `spvi_2` executable
// (src/spvi_2.cu main, :730-796), built on the C ABI.
//
// Reads temp_modelOp_dirName.txt (5 lines: prob_type, prob_name, prob_specs,
// alpha, model path), loads the model in the reference's layout, runs value
// iteration and writes data_solverOutput/<type>/<name>/<specs>/[<alpha>/]
// policy.npy (uint32, (Ns,1)) and value_function.npy (float32, (Ns,1)).
// Default: Jacobi sweeps to a sup-norm below 0.1 (the reference's
// s_stopping_thresh, :757).  Environment: E2E_VI_THRESHOLD overrides the
// threshold; E2E_VI_METHOD=layered uses the one-sweep backward schedule.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

#include "e2e_dp.h"
#include "npy_io.h"

namespace fs = std::filesystem;

int main() {
  std::ifstream path_file("temp_modelOp_dirName.txt");
  if (!path_file) {
    std::fprintf(stderr, "spvi_2: temp_modelOp_dirName.txt not found\n");
    return 2;
  }
  std::string prob_type, prob_name, prob_specs, alpha_str, model_path;
  std::getline(path_file, prob_type);
  std::getline(path_file, prob_name);
  std::getline(path_file, prob_specs);
  std::getline(path_file, alpha_str);
  std::getline(path_file, model_path);
  std::string results = "data_solverOutput/" + prob_type + "/" + prob_name + "/" + prob_specs + "/";
  if (prob_type == "custom1") results += "/" + alpha_str + "/";
  std::error_code ec;
  fs::create_directories(results, ec);

  e2e_vi_opts o{};
  o.method = 0;
  o.threshold = 0.1f;
  if (const char* t = std::getenv("E2E_VI_THRESHOLD")) o.threshold = std::strtof(t, nullptr);
  if (const char* mth = std::getenv("E2E_VI_METHOD")) o.method = std::string(mth) == "layered" ? 1 : 0;

  auto t0 = std::chrono::steady_clock::now();
  e2e_model* m = nullptr;
  e2e_status st = e2e_model_read_npy(model_path.c_str(), &m, nullptr);
  if (st != E2E_OK) {
    std::fprintf(stderr, "spvi_2: %s: %s\n", e2e_status_string(st), e2e_last_error());
    return 3;
  }
  e2e_model_info info;
  e2e_model_get_info(m, &info);
  std::vector<int32_t> policy((size_t)info.ns);
  std::vector<float> value((size_t)info.ns);
  e2e_vi_stats stats{};
  st = e2e_spvi_solve(m, &o, policy.data(), value.data(), E2E_HOST, &stats, nullptr);
  auto t1 = std::chrono::steady_clock::now();
  e2e_model_free(m);
  if (st != E2E_OK) {
    std::fprintf(stderr, "spvi_2: %s: %s\n", e2e_status_string(st), e2e_last_error());
    return 4;
  }
  std::printf("num_iterations%d\n", stats.iterations);
  std::printf("final sup norm = %g\n", stats.residual);
  std::printf("---- total solve time = %.6f\n", std::chrono::duration<double>(t1 - t0).count());
  std::string err;
  const std::vector<size_t> shp{(size_t)info.ns, 1};
  if (!e2e::npy::write(results + "policy.npy", "<u4", shp, policy.data(), err) ||
      !e2e::npy::write(results + "value_function.npy", "<f4", shp, value.data(), err)) {
    std::fprintf(stderr, "spvi_2: %s\n", err.c_str());
    return 5;
  }
  std::printf("saved policy and value function to %s\n", results.c_str());
  return 0;
}
