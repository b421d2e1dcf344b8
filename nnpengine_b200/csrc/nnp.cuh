// Network-term state shared by the FP32 (nnp.cu) and BF16 tensor-core (nnp_tc.cu) paths.
#pragma once
#include <vector>

#include "internal.cuh"

struct NnpTc;   // tcgen05 path state (nnp_tc.cu)

struct NnpModel {
  int kind = 1;              // 0 gauss (reference tables), 1 radial embedding
  float rc = 6.f, scale = 1.f;
  int nbin = 0, e1 = 32, e2 = 64, din = 256, h1 = 128, h2 = 128, ntype = 0, npair = 0;
  int cap6 = 256;
  bool bf16 = false;
  bool g_bf16 = false;       // d_G holds BF16 rows [N][din] (the tensor-core path's descriptor)
  bool enabled = true;
  float* d_embw = nullptr;   // per species: W1[e1] b1[e1] W2[e1][e2] b2[e2]
  float* d_fitw = nullptr;   // per species: A1[din][h1] c1 A2[h1][h2] c2 A3[h2] c3
  float* d_fitg = nullptr;   // per species, 16-byte aligned parts: A1 A2 A2^T A1^T c1 c2 A3 (FP32 GEMMs)
  size_t fitg_block = 0;     // floats per species in d_fitg
  float2* d_tdesc = nullptr; // gauss: (desc, f_desc) [npair][80][nbin+1]
  float2* d_tpair = nullptr; // gauss: (U, F/r) [npair][4][nbin+1]
  float *d_G = nullptr, *d_dG = nullptr;   // [N][din] sorted order
  double* d_enet = nullptr;                // network energy per atom
  uint32_t* d_list6 = nullptr;             // pairs inside rc, [N][cap6]
  int* d_n6 = nullptr;
  int *d_sidx = nullptr, *d_scount = nullptr, *d_soff_dev = nullptr;
  std::vector<int> soff;                   // species row offsets
  float *d_H1 = nullptr, *d_G2 = nullptr, *d_G1 = nullptr;
  std::vector<float> h_embw, h_fitw;
  std::vector<float2> h_tpair;
  NnpTc* tc = nullptr;
};

struct NnpArgs {
  const float4* pos;
  const int2* info;
  const int* pairtype;
  const int* gowner;
  const uint32_t* list6;
  const int* n6;
  int cap6, ntype, N, nbin, e2;
  float r_dr, rc, scale;
  const float2* tdesc;
  const float2* tpair;
  const float* embw;
  float* G;
  float* dG;
  float4* frc;
  double* eatom;
  double* watom;
};

int nnp_tc_setup(nnpe_ctx* c);
void nnp_tc_free(NnpModel* m);
int nnp_tc_forces_enqueue(nnpe_ctx* c, bool ev);
int nnp_tc_autotune(nnpe_ctx* c, int reps, bool use_cache, int* grid_desc, int* grid_force);
int nnp_tc_set_grids(nnpe_ctx* c, int grid_desc, int grid_force);
int nnp_tc_get_grids(nnpe_ctx* c, int* grid_desc, int* grid_force);
