// Model files in the reference's on-disk layout.
//
// Writer: save_master_Coos_to_file (src/build_model.cu:1246-1314) concatenates
// the per-action COO vectors action-major (for a: for t: for cell: S2
// ascending), shifts S1 by a*Ns, lays R out as [a][s] with a zero last layer,
// and saves DP_relv_params = [Ns, Na] (int64) and prob_params (32 floats).
// Reader: get_mdp_model (src/spvi_2.cu:393-504) loads the same files (S1/S2 as
// int32 after src/convert_model_datatype.py:19-23 ran).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "e2e_dp.h"
#include "internal.h"
#include "npy_io.h"

using namespace e2e;

#define CK(call)                                          \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return cuda_fail(_e, #call);   \
  } while (0)

extern "C" e2e_status e2e_model_write_npy(const e2e_model* m, const e2e_problem* p,
                                          const char* dir, int index_bits) {
  if (!m || !dir) return fail(E2E_ERR_INVALID, "null argument");
  if (index_bits != 32 && index_bits != 64) return fail(E2E_ERR_INVALID, "index_bits must be 32 or 64");
  const e2e_problem* pp = p ? p : (m->has_prob ? &m->prob : nullptr);
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  const int64_t nnz = m->nnz, ns = m->ns, na = m->na;
  std::vector<int64_t> rp((size_t)m->n_rows + 1);
  std::vector<int32_t> col((size_t)std::max<int64_t>(nnz, 1));
  std::vector<uint32_t> cnt((size_t)std::max<int64_t>(nnz, 1));
  std::vector<float> R((size_t)(ns * na));
  e2e_status s = e2e_model_copy_to_host(m, rp.data(), col.data(), cnt.data(), R.data(), nullptr);
  if (s != E2E_OK) return s;
  std::vector<int64_t> S1_64, S2_64;
  std::vector<int32_t> S1_32, S2_32;
  if (index_bits == 64) {
    S1_64.resize((size_t)nnz);
    S2_64.resize((size_t)nnz);
  } else {
    if (na * ns > INT32_MAX) return fail(E2E_ERR_UNSUPPORTED, "S1 does not fit int32");
    S1_32.resize((size_t)nnz);
    S2_32.resize((size_t)nnz);
  }
  std::vector<float> val((size_t)nnz);
  const float fn = (float)m->nrzns;
  int64_t o = 0;
  for (int64_t a = 0; a < na; ++a) {
    for (int64_t st = 0; st < m->n_row_states; ++st) {
      const int64_t row = st * na + a;
      for (int64_t k = rp[row]; k < rp[row + 1]; ++k) {
        const int64_t s1 = a * ns + st;
        if (index_bits == 64) {
          S1_64[o] = s1;
          S2_64[o] = col[k];
        } else {
          S1_32[o] = (int32_t)s1;
          S2_32[o] = col[k];
        }
        if (m->count_type == E2E_VALUE_F32) {
          float v;
          std::memcpy(&v, &cnt[k], 4);
          val[o] = v;
        } else {
          val[o] = (float)cnt[k] / fn;  // reduce_kernel: count/nrzns, src/build_model.cu:637
        }
        ++o;
      }
    }
  }
  std::vector<float> Rref((size_t)(ns * na));
  for (int64_t a = 0; a < na; ++a)
    for (int64_t st = 0; st < ns; ++st) Rref[a * ns + st] = R[st * na + a];
  const std::string d = std::string(dir) + "/";
  std::string err;
  const std::vector<size_t> shp{(size_t)nnz, 1};
  bool ok = true;
  if (index_bits == 64) {
    ok = ok && npy::write(d + "master_cooS1.npy", "<i8", shp, S1_64.data(), err);
    ok = ok && npy::write(d + "master_cooS2.npy", "<i8", shp, S2_64.data(), err);
  } else {
    ok = ok && npy::write(d + "master_cooS1.npy", "<i4", shp, S1_32.data(), err);
    ok = ok && npy::write(d + "master_cooS2.npy", "<i4", shp, S2_32.data(), err);
  }
  ok = ok && npy::write(d + "master_cooVal.npy", "<f4", shp, val.data(), err);
  ok = ok && npy::write(d + "master_R.npy", "<f4", {(size_t)(ns * na), 1}, Rref.data(), err);
  int64_t dp[2] = {ns, na};
  ok = ok && npy::write(d + "DP_relv_params.npy", "<i8", {2, 1}, dp, err);
  if (pp) {
    float params[32];
    e2e_problem_to_params(pp, params);
    ok = ok && npy::write(d + "prob_params.npy", "<f4", {32, 1}, params, err);
  }
  if (!ok) return fail(E2E_ERR_IO, err);
  return E2E_OK;
}

static bool load_int_column(const npy::Array& a, std::vector<int64_t>& out, std::string& err) {
  const size_t n = a.count();
  out.resize(n);
  if (a.kind() == 'i' && a.word() == 4) {
    const int32_t* p = a.as<int32_t>();
    for (size_t i = 0; i < n; ++i) out[i] = p[i];
  } else if (a.kind() == 'i' && a.word() == 8) {
    std::memcpy(out.data(), a.data.data(), n * 8);
  } else if (a.kind() == 'u' && a.word() == 4) {
    const uint32_t* p = a.as<uint32_t>();
    for (size_t i = 0; i < n; ++i) out[i] = p[i];
  } else {
    err = "unsupported index dtype " + a.descr;
    return false;
  }
  return true;
}

extern "C" e2e_status e2e_model_read_npy(const char* dir, e2e_model** out, void* stream) {
  if (!dir || !out) return fail(E2E_ERR_INVALID, "null argument");
  *out = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  const std::string d = std::string(dir) + "/";
  npy::Array aS1, aS2, aV, aR, aDP, aPP;
  std::string err;
  if (!npy::read(d + "master_cooS1.npy", aS1, err) || !npy::read(d + "master_cooS2.npy", aS2, err) ||
      !npy::read(d + "master_cooVal.npy", aV, err) || !npy::read(d + "master_R.npy", aR, err) ||
      !npy::read(d + "DP_relv_params.npy", aDP, err))
    return fail(E2E_ERR_IO, err);
  bool have_pp = npy::read(d + "prob_params.npy", aPP, err);
  std::vector<int64_t> S1, S2, DP;
  if (!load_int_column(aS1, S1, err) || !load_int_column(aS2, S2, err) || !load_int_column(aDP, DP, err))
    return fail(E2E_ERR_IO, err);
  if (DP.size() < 2) return fail(E2E_ERR_IO, "DP_relv_params must hold [Ns, Na]");
  if (aV.kind() != 'f' || aV.word() != 4 || aR.kind() != 'f' || aR.word() != 4)
    return fail(E2E_ERR_IO, "master_cooVal and master_R must be float32");
  const int64_t ns = DP[0], na = DP[1];
  const int64_t nnz = (int64_t)S1.size();
  if (ns <= 0 || na <= 0 || na > 32) return fail(E2E_ERR_UNSUPPORTED, "Na must be in 1..32");
  if ((int64_t)S2.size() != nnz || (int64_t)aV.count() != nnz)
    return fail(E2E_ERR_IO, "S1, S2 and Val lengths differ");
  if ((int64_t)aR.count() != ns * na) return fail(E2E_ERR_IO, "master_R must hold Ns*Na values");
  const float* val = aV.as<float>();
  const float* Rref = aR.as<float>();
  std::vector<int64_t> rp((size_t)(ns * na) + 1, 0);
  for (int64_t k = 0; k < nnz; ++k) {
    if (S1[k] < 0 || S1[k] >= ns * na || S2[k] < 0 || S2[k] >= ns)
      return fail(E2E_ERR_IO, "row or column index out of range");
    const int64_t a = S1[k] / ns, s = S1[k] % ns;
    rp[(size_t)(s * na + a) + 1]++;
  }
  for (size_t r = 1; r < rp.size(); ++r) rp[r] += rp[r - 1];
  std::vector<int64_t> fill(rp.begin(), rp.end() - 1);
  std::vector<int32_t> col((size_t)std::max<int64_t>(nnz, 1));
  std::vector<float> v((size_t)std::max<int64_t>(nnz, 1));
  for (int64_t k = 0; k < nnz; ++k) {
    const int64_t a = S1[k] / ns, s = S1[k] % ns;
    const int64_t pos = fill[(size_t)(s * na + a)]++;
    col[(size_t)pos] = (int32_t)S2[k];
    v[(size_t)pos] = val[k];
  }
  e2e_model* m = new e2e_model();
  m->ns = ns;
  m->na = (int32_t)na;
  m->n_row_states = ns;
  m->n_rows = ns * na;
  m->nnz = nnz;
  m->nrzns = 1;
  m->count_type = E2E_VALUE_F32;
  if (have_pp && aPP.kind() == 'f' && aPP.word() == 4 && aPP.count() >= 20) {
    e2e_problem_from_params(aPP.as<float>(), &m->prob);
    m->has_prob = true;
    const int32_t nr = m->prob.nrzns;
    bool counts = nr > 0 && nr < 65536;
    for (int64_t k = 0; counts && k < nnz; ++k) {
      double c = std::rint((double)v[(size_t)k] * nr);
      if (c < 1 || c > nr || (float)c / (float)nr != v[(size_t)k]) counts = false;
    }
    if (counts) {
      m->nrzns = nr;
      m->count_type = E2E_COUNT_U16;
    }
    const int64_t g = m->prob.gsize, nt = m->prob.nt;
    if (g > 0 && nt > 0 && g * g * nt == ns) {
      m->ncells = (int32_t)(g * g);
      m->nt = (int32_t)nt;
      bool layered = true;
      for (int64_t r = 0; layered && r < ns * na; ++r) {
        const int64_t s = r / na, t = s / (g * g);
        for (int64_t k = rp[(size_t)r]; k < rp[(size_t)r + 1]; ++k)
          if (col[(size_t)k] / (g * g) != t + 1) {
            layered = false;
            break;
          }
      }
      m->layered = layered;
    }
  }
  m->index_bits = nnz < ((int64_t)1 << 31) ? 32 : 64;
  std::vector<float> Rsa((size_t)(ns * na));
  for (int64_t a = 0; a < na; ++a)
    for (int64_t s = 0; s < ns; ++s) Rsa[(size_t)(s * na + a)] = Rref[a * ns + s];
  auto cleanup = [&](e2e_status code, cudaError_t e, const char* what) {
    free_model_buffers(m);
    delete m;
    return e == cudaSuccess ? code : cuda_fail(e, what);
  };
  cudaError_t e;
  const size_t pb = m->index_bits == 32 ? 4 : 8;
  if ((e = dalloc(&m->row_ptr, pb * rp.size(), st)) != cudaSuccess) return cleanup(E2E_OK, e, "alloc(row_ptr)");
  if ((e = dalloc((void**)&m->col, 4 * (col.size() + 16), st)) != cudaSuccess) return cleanup(E2E_OK, e, "alloc(col)");
  if ((e = dalloc((void**)&m->R, 4 * Rsa.size(), st)) != cudaSuccess) return cleanup(E2E_OK, e, "alloc(R)");
  if (m->index_bits == 32) {
    std::vector<int32_t> rp32(rp.begin(), rp.end());
    e = cudaMemcpyAsync(m->row_ptr, rp32.data(), 4 * rp32.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  } else {
    e = cudaMemcpyAsync(m->row_ptr, rp.data(), 8 * rp.size(), cudaMemcpyHostToDevice, st);
  }
  if (e != cudaSuccess) return cleanup(E2E_OK, e, "upload row_ptr");
  if ((e = cudaMemcpyAsync(m->col, col.data(), 4 * col.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return cleanup(E2E_OK, e, "upload col");
  if ((e = cudaMemcpyAsync(m->R, Rsa.data(), 4 * Rsa.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return cleanup(E2E_OK, e, "upload R");
  if (m->count_type == E2E_COUNT_U16) {
    std::vector<uint16_t> c16((size_t)std::max<int64_t>(nnz, 1));
    for (int64_t k = 0; k < nnz; ++k) c16[(size_t)k] = (uint16_t)std::rint((double)v[(size_t)k] * m->nrzns);
    if ((e = dalloc(&m->cnt, 2 * (c16.size() + 16), st)) != cudaSuccess) return cleanup(E2E_OK, e, "alloc(cnt)");
    e = cudaMemcpyAsync(m->cnt, c16.data(), 2 * c16.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  } else {
    if ((e = dalloc(&m->cnt, 4 * (v.size() + 16), st)) != cudaSuccess) return cleanup(E2E_OK, e, "alloc(cnt)");
    e = cudaMemcpyAsync(m->cnt, v.data(), 4 * v.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e != cudaSuccess) return cleanup(E2E_OK, e, "upload counts");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cleanup(E2E_OK, e, "sync");
  *out = m;
  return E2E_OK;
}
