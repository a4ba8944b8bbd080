// Drop-in replacement for the reference's `build_model` executable
// (src/build_model.cu main, :926-1238), built on the C ABI.
//
// Same command line (`build_model [ALPHA*100]`), same inputs
// (data_input/<prob_name>/{all_u_mat,all_v_mat,all_ui_mat,all_vi_mat,all_Yi,
// all_s_mat,obstacle_mask}.npy), same outputs (data_modelOutput/<prob_type>/
// <prob_name>/<prob_specs>/[<alpha>/] with master_cooS1/S2 (int64),
// master_cooVal, master_R, DP_relv_params, prob_params) and the same
// temp_modelOp_dirName.txt hand-off file.  The problem is read at run time from
// input_to_build_model.h in the working directory (or $E2E_CONFIG_HEADER).
#include <chrono>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

#include "config_header.h"
#include "e2e_dp.h"
#include "npy_io.h"

namespace fs = std::filesystem;

static int get_reward_type(const std::string& t) {  // src/build_model.cu:898-918
  if (t == "time") return 0;
  if (t == "energy1") return 1;
  if (t == "energy2") return 2;
  if (t == "energy3") return 3;
  if (t == "custom1") return 4;
  return -1;
}

static bool load(const std::string& path, const char* kind, size_t expect, e2e::npy::Array& a) {
  std::string err;
  if (!e2e::npy::read(path, a, err)) {
    std::fprintf(stderr, "build_model: %s\n", err.c_str());
    return false;
  }
  if (a.kind() != kind[0] || a.word() != 4) {
    std::fprintf(stderr, "build_model: %s must be %s32\n", path.c_str(), kind[0] == 'f' ? "float" : "int");
    return false;
  }
  if (a.count() != expect) {
    std::fprintf(stderr, "build_model: %s has %zu elements, expected %zu\n", path.c_str(), a.count(), expect);
    return false;
  }
  return true;
}

int main(int argc, char** argv) {
  const char* hp = std::getenv("E2E_CONFIG_HEADER");
  std::string header_path = hp ? hp : "input_to_build_model.h";
  e2e::cfg::Header H;
  try {
    H.parse_file(header_path);
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "build_model: %s\n", ex.what());
    return 2;
  }
  try {
    const std::string prob_type = H.str("prob_type");
    const std::string prob_name = H.str("prob_name");
    float alpha = (float)H.num("alpha_header");
    if (argc > 1) alpha = std::stof(argv[1]) / 100;  // :936-943
    const int reward_type = get_reward_type(prob_type);
    if (reward_type < 0) {
      std::fprintf(stderr, "build_model: unknown prob_type %s\n", prob_type.c_str());
      return 2;
    }
    e2e_problem p{};
    p.gsize = (int32_t)H.num("gsize");
    p.num_ac_speeds = (int32_t)H.num("num_ac_speeds");
    p.num_ac_angles = (int32_t)H.num("num_ac_angles");
    p.num_actions = p.num_ac_speeds * p.num_ac_angles;
    p.nrzns = (int32_t)H.num("nrzns");
    p.F = (float)H.num("F");
    p.dt = (float)H.num("dt");
    p.r_outbound = (float)H.num("r_outbound");
    p.r_terminal = (float)H.num("r_terminal");
    p.nmodes = (int32_t)H.num("nmodes");
    p.i_term = (int32_t)H.num("i_term");
    p.j_term = (int32_t)H.num("j_term");
    p.nt = (int32_t)H.num("nt");
    p.is_stationary = H.has("is_stationary") ? (int32_t)H.num("is_stationary") : 0;
    p.term_subgrid_size = (int32_t)H.num("term_subgrid_size");
    p.reward_type = reward_type;
    p.dx = (float)H.num("dx");
    p.dy = H.has("dy") ? (float)H.num("dy") : p.dx;
    p.neighb_gsize = (int32_t)H.num("neighb_gsize");
    p.alpha = alpha;
    p.x0 = H.has("x0") ? (float)H.num("x0") : p.dx / 2;
    p.y0 = H.has("y0") ? (float)H.num("y0") : p.dy / 2;

    // output paths and the hand-off file, :953-975
    const std::string prob_specs = "a" + std::to_string(p.num_ac_speeds) + "x" +
                                   std::to_string(p.num_ac_angles) + "_i" + std::to_string(p.i_term) +
                                   "_j" + std::to_string(p.j_term) + "_ref" +
                                   std::to_string(p.term_subgrid_size);
    std::string op = "data_modelOutput/" + prob_type + "/" + prob_name + "/" + prob_specs + "/";
    if (reward_type > 3) op += std::to_string(alpha) + "/";
    std::error_code ec;
    fs::create_directories(op, ec);
    {
      std::ofstream fout("temp_modelOp_dirName.txt");
      fout << prob_type << "\n" << prob_name << "\n" << prob_specs << "\n" << std::to_string(alpha) << "\n" << op;
    }

    // inputs, :978-1019
    const std::string d = "data_input/" + prob_name + "/";
    const size_t nc = (size_t)p.gsize * p.gsize, nt = (size_t)p.nt, nm = (size_t)p.nmodes;
    e2e::npy::Array u, v, ui, vi, yi, s, mask;
    if (!load(d + "all_u_mat.npy", "f", nt * nc, u) || !load(d + "all_v_mat.npy", "f", nt * nc, v) ||
        !load(d + "all_ui_mat.npy", "f", nt * nm * nc, ui) ||
        !load(d + "all_vi_mat.npy", "f", nt * nm * nc, vi) ||
        !load(d + "all_Yi.npy", "f", nt * (size_t)p.nrzns * nm, yi) ||
        !load(d + "all_s_mat.npy", "f", nt * nc, s) || !load(d + "obstacle_mask.npy", "i", nt * nc, mask))
      return 3;
    e2e_fields f{u.as<float>(), v.as<float>(), ui.as<float>(), vi.as<float>(), yi.as<float>(),
                 s.as<float>(), mask.as<int32_t>()};
    auto t0 = std::chrono::steady_clock::now();
    e2e_model* m = nullptr;
    e2e_status st = e2e_build_model(&p, &f, E2E_HOST, nullptr, &m, nullptr);
    if (st != E2E_OK) {
      std::fprintf(stderr, "build_model: %s: %s\n", e2e_status_string(st), e2e_last_error());
      return 4;
    }
    auto t1 = std::chrono::steady_clock::now();
    st = e2e_model_write_npy(m, &p, op.c_str(), 64);
    auto t2 = std::chrono::steady_clock::now();
    e2e_model_info info;
    e2e_model_get_info(m, &info);
    e2e_model_free(m);
    if (st != E2E_OK) {
      std::fprintf(stderr, "build_model: %s: %s\n", e2e_status_string(st), e2e_last_error());
      return 5;
    }
    std::printf("build time = %.6f sec\n", std::chrono::duration<double>(t1 - t0).count());
    std::printf("save time = %.6f sec\n", std::chrono::duration<double>(t2 - t1).count());
    std::printf("Ns = %lld, Na = %d, nnz = %lld, dropped samples = %llu\n", (long long)info.ns,
                info.num_actions, (long long)info.nnz, (unsigned long long)info.dropped);
    std::printf("saved files to %s\n", op.c_str());
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "build_model: %s\n", ex.what());
    return 2;
  }
  return 0;
}
