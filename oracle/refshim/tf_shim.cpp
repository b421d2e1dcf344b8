// Test infrastructure only (the oracle's network stand-in; never linked into the product).
//
// Implements the TensorFlow C-API calls made by the reference's TFCALL (pair_nnp.cpp:12-119)
// so that NNPOTENTIAL_TBL (pair_nnp.cpp:433-793) runs unmodified. TF_LoadSessionFromSavedModel
// receives the first token of the NNP paramfile (pair_nnp.cpp:458); here that token names an
// NNPE model file (text header, "end" line, then little-endian float32 weights). TF_SessionRun
// evaluates the per-atom fitting network of that file in double precision on the descriptor
// tensor [nmol, NUM_ATOM, 20] and returns E (scalar) and dE/dG (same shape as the input), the
// two outputs NNPOTENTIAL_TBL reads (pair_nnp.cpp:697-706, run.cpp:1253).
#include "tensorflow/c/c_api.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

struct TF_Graph { int dummy; };
struct TF_Status { TF_Code code; std::string msg; };
struct TF_SessionOptions { int dummy; };
struct TF_Operation { std::string name; };
struct TF_Buffer { int dummy; };
struct TF_Tensor {
  TF_DataType dtype;
  std::vector<int64_t> dims;
  std::vector<unsigned char> data;
};

namespace {
struct FitNet {
  int din = 0, h1 = 0, h2 = 0, ntype = 0;
  std::vector<int> slot_type;           // per atom slot of the molecule
  std::vector<std::vector<double>> A1, c1, A2, c2, A3, c3;  // per type
  // float copies for the timing build (TF evaluates the reference's network in float): the
  // weights as read and transposed, so that every loop below runs along contiguous memory
  std::vector<std::vector<float>> fA1, fc1, fA2, fc2, fA3, fA1T, fA2T;
};
}  // namespace

struct TF_Session { FitNet net; std::vector<TF_Operation*> ops; };

static void set_status(TF_Status* s, TF_Code c, const std::string& m) {
  if (s) { s->code = c; s->msg = m; }
}

extern "C" {

TF_Graph* TF_NewGraph(void) { return new TF_Graph(); }
void TF_DeleteGraph(TF_Graph* g) { delete g; }
TF_Status* TF_NewStatus(void) { auto* s = new TF_Status(); s->code = TF_OK; return s; }
void TF_DeleteStatus(TF_Status* s) { delete s; }
TF_Code TF_GetCode(const TF_Status* s) { return s->code; }
const char* TF_Message(const TF_Status* s) { return s->msg.c_str(); }
TF_SessionOptions* TF_NewSessionOptions(void) { return new TF_SessionOptions(); }
void TF_DeleteSessionOptions(TF_SessionOptions* o) { delete o; }
void TF_SetConfig(TF_SessionOptions*, const void*, size_t, TF_Status* s) { set_status(s, TF_OK, ""); }

static TF_Session* g_last_session = nullptr;

TF_Session* TF_LoadSessionFromSavedModel(const TF_SessionOptions*, const TF_Buffer*,
                                         const char* export_dir, const char* const*, int,
                                         TF_Graph*, TF_Buffer*, TF_Status* st) {
  FILE* fp = fopen(export_dir, "rb");
  if (!fp) { set_status(st, TF_INVALID_ARGUMENT, std::string("cannot open model ") + export_dir); return nullptr; }
  auto* sess = new TF_Session();
  FitNet& n = sess->net;
  char line[512];
  std::string desc;
  int npair = 0;
  while (fgets(line, sizeof line, fp)) {
    char key[64];
    if (sscanf(line, "%63s", key) != 1) continue;
    std::string k(key);
    if (k == "end") break;
    if (k == "descriptor") { char d[64]; int a = 0; sscanf(line, "%*s %63s %d", d, &a); desc = d; if (desc == "gauss") n.din = a; }
    else if (k == "fitting") sscanf(line, "%*s %d %d", &n.h1, &n.h2);
    else if (k == "ntype") sscanf(line, "%*s %d", &n.ntype);
    else if (k == "npair") sscanf(line, "%*s %d", &npair);
    else if (k == "slots") {
      int cnt = 0, off = 0, used = 0;
      sscanf(line, "%*s %d%n", &cnt, &off);
      n.slot_type.resize(cnt);
      for (int i = 0; i < cnt; ++i) { sscanf(line + off, "%d%n", &n.slot_type[i], &used); off += used; }
    }
  }
  if (desc != "gauss" || n.din <= 0 || n.h1 <= 0 || n.h2 <= 0 || n.ntype <= 0) {
    fclose(fp); delete sess;
    set_status(st, TF_INVALID_ARGUMENT, "model is not a gauss-descriptor fitting network");
    return nullptr;
  }
  auto rd = [&](std::vector<double>& v, size_t cnt) {
    std::vector<float> tmp(cnt);
    if (fread(tmp.data(), sizeof(float), cnt, fp) != cnt) return false;
    v.assign(tmp.begin(), tmp.end());
    return true;
  };
  n.A1.resize(n.ntype); n.c1.resize(n.ntype); n.A2.resize(n.ntype); n.c2.resize(n.ntype);
  n.A3.resize(n.ntype); n.c3.resize(n.ntype);
  bool ok = true;
  for (int t = 0; t < n.ntype && ok; ++t)
    ok = rd(n.A1[t], (size_t)n.din * n.h1) && rd(n.c1[t], n.h1) && rd(n.A2[t], (size_t)n.h1 * n.h2) &&
         rd(n.c2[t], n.h2) && rd(n.A3[t], n.h2) && rd(n.c3[t], 1);
  fclose(fp);
  if (!ok) { delete sess; set_status(st, TF_INVALID_ARGUMENT, "truncated model weights"); return nullptr; }
  n.fA1.resize(n.ntype); n.fc1.resize(n.ntype); n.fA2.resize(n.ntype); n.fc2.resize(n.ntype);
  n.fA3.resize(n.ntype); n.fA1T.resize(n.ntype); n.fA2T.resize(n.ntype);
  for (int t = 0; t < n.ntype; ++t) {
    n.fA1[t].assign(n.A1[t].begin(), n.A1[t].end()); n.fc1[t].assign(n.c1[t].begin(), n.c1[t].end());
    n.fA2[t].assign(n.A2[t].begin(), n.A2[t].end()); n.fc2[t].assign(n.c2[t].begin(), n.c2[t].end());
    n.fA3[t].assign(n.A3[t].begin(), n.A3[t].end());
    n.fA1T[t].resize((size_t)n.din * n.h1); n.fA2T[t].resize((size_t)n.h1 * n.h2);
    for (int d = 0; d < n.din; ++d)
      for (int k = 0; k < n.h1; ++k) n.fA1T[t][(size_t)k * n.din + d] = (float)n.A1[t][(size_t)d * n.h1 + k];
    for (int k = 0; k < n.h1; ++k)
      for (int m = 0; m < n.h2; ++m) n.fA2T[t][(size_t)m * n.h1 + k] = (float)n.A2[t][(size_t)k * n.h2 + m];
  }
  set_status(st, TF_OK, "");
  g_last_session = sess;
  return sess;
}

TF_Operation* TF_GraphOperationByName(TF_Graph*, const char* name) {
  auto* op = new TF_Operation();
  op->name = name;
  return op;
}

TF_Tensor* TF_AllocateTensor(TF_DataType dt, const int64_t* dims, int nd, size_t len) {
  auto* t = new TF_Tensor();
  t->dtype = dt;
  t->dims.assign(dims, dims + nd);
  t->data.assign(len, 0);
  return t;
}
void* TF_TensorData(const TF_Tensor* t) { return (void*)t->data.data(); }
void TF_DeleteTensor(TF_Tensor* t) { delete t; }

void TF_SessionRun(TF_Session* session, const TF_Buffer*, const TF_Output*, TF_Tensor* const* input_values,
                   int ninputs, const TF_Output*, TF_Tensor** output_values, int noutputs,
                   const TF_Operation* const*, int, TF_Buffer*, TF_Status* st) {
  if (!session || ninputs < 1 || noutputs < 2) { set_status(st, TF_INVALID_ARGUMENT, "bad session run"); return; }
  const FitNet& n = session->net;
  const TF_Tensor* in = input_values[0];
  size_t nval = in->data.size() / sizeof(float);
  size_t natom = nval / n.din;
  const float* G = (const float*)in->data.data();
  int64_t dimE = 1;
  TF_Tensor* tE = TF_AllocateTensor(TF_FLOAT, &dimE, 0, sizeof(float));
  TF_Tensor* tD = TF_AllocateTensor(TF_FLOAT, in->dims.data(), (int)in->dims.size(), in->data.size());
  float* dG = (float*)tD->data.data();
  double E = 0;
  const int nslot = (int)n.slot_type.size();
#ifdef SHIM_FLOAT
  // Timing build: the network in float, as TF runs the reference's model, serial, as the
  // reference configures its TF session (intra/inter-op threads 1, pair_nnp.cpp:23-24); every
  // inner loop runs along contiguous weights so that the compiler vectorises it.
  {
    std::vector<float> h1(n.h1), h2(n.h2), g1(n.h1), g2(n.h2);
    for (long a = 0; a < (long)natom; ++a) {
      const int t = n.slot_type[a % nslot];
      const float* g = G + a * n.din;
      const float *A1 = n.fA1[t].data(), *c1 = n.fc1[t].data(), *A2 = n.fA2[t].data(), *c2 = n.fc2[t].data();
      const float *A3 = n.fA3[t].data(), *A1T = n.fA1T[t].data(), *A2T = n.fA2T[t].data();
      for (int k = 0; k < n.h1; ++k) h1[k] = c1[k];
      for (int d = 0; d < n.din; ++d) {
        const float gd = g[d];
        const float* row = A1 + (size_t)d * n.h1;
        for (int k = 0; k < n.h1; ++k) h1[k] += gd * row[k];
      }
      for (int k = 0; k < n.h1; ++k) h1[k] = std::tanh(h1[k]);
      for (int m = 0; m < n.h2; ++m) h2[m] = c2[m];
      for (int k = 0; k < n.h1; ++k) {
        const float hk = h1[k];
        const float* row = A2 + (size_t)k * n.h2;
        for (int m = 0; m < n.h2; ++m) h2[m] += hk * row[m];
      }
      float e = (float)n.c3[t][0];
      for (int m = 0; m < n.h2; ++m) {
        h2[m] = std::tanh(h2[m]);
        e += h2[m] * A3[m];
        g2[m] = A3[m] * (1 - h2[m] * h2[m]);
      }
      E += e;
      for (int k = 0; k < n.h1; ++k) g1[k] = 0;
      for (int m = 0; m < n.h2; ++m) {
        const float gm = g2[m];
        const float* row = A2T + (size_t)m * n.h1;
        for (int k = 0; k < n.h1; ++k) g1[k] += gm * row[k];
      }
      for (int k = 0; k < n.h1; ++k) g1[k] *= 1 - h1[k] * h1[k];
      float* out = dG + a * n.din;
      for (int d = 0; d < n.din; ++d) out[d] = 0;
      for (int k = 0; k < n.h1; ++k) {
        const float gk = g1[k];
        const float* row = A1T + (size_t)k * n.din;
        for (int d = 0; d < n.din; ++d) out[d] += gk * row[d];
      }
    }
  }
  if (false)
#endif
  // serial, as the reference configures its TF session (intra/inter-op threads 1, pair_nnp.cpp:23-24)
  for (long a = 0; a < (long)natom; ++a) {
    std::vector<double> h1(n.h1), h2(n.h2), g1(n.h1), g2(n.h2);
    const int t = n.slot_type[a % nslot];
    const float* g = G + a * n.din;
    const std::vector<double>&A1 = n.A1[t], &c1 = n.c1[t], &A2 = n.A2[t], &c2 = n.c2[t], &A3 = n.A3[t];
    for (int k = 0; k < n.h1; ++k) {
      double z = c1[k];
      for (int d = 0; d < n.din; ++d) z += (double)g[d] * A1[(size_t)d * n.h1 + k];
      h1[k] = std::tanh(z);
    }
    double e = n.c3[t][0];
    for (int m = 0; m < n.h2; ++m) {
      double z = c2[m];
      for (int k = 0; k < n.h1; ++k) z += h1[k] * A2[(size_t)k * n.h2 + m];
      h2[m] = std::tanh(z);
      e += h2[m] * A3[m];
    }
    E += e;
    for (int m = 0; m < n.h2; ++m) g2[m] = A3[m] * (1 - h2[m] * h2[m]);
    for (int k = 0; k < n.h1; ++k) {
      double s = 0;
      for (int m = 0; m < n.h2; ++m) s += A2[(size_t)k * n.h2 + m] * g2[m];
      g1[k] = s * (1 - h1[k] * h1[k]);
    }
    for (int d = 0; d < n.din; ++d) {
      double s = 0;
      for (int k = 0; k < n.h1; ++k) s += A1[(size_t)d * n.h1 + k] * g1[k];
      dG[a * n.din + d] = (float)s;
    }
  }
  *(float*)tE->data.data() = (float)E;
  output_values[0] = tE;
  output_values[1] = tD;
  for (int i = 2; i < noutputs; ++i) output_values[i] = TF_AllocateTensor(TF_FLOAT, &dimE, 0, sizeof(float));
  set_status(st, TF_OK, "");
}

}  // extern "C"
