// lt_api.cuh -- cuBLASLt entry points resolved with dlopen at first use, so
// librotormap_b200.so has no link-time dependency on the library.  Used by
// the plain batch path (fp8 GEMM) and the FP64 check (fp64 GEMM).
#pragma once

#include <cublasLt.h>

namespace r2m {

struct LtApi {
  void *so = nullptr;
  decltype(&cublasLtCreate) create;
  decltype(&cublasLtDestroy) destroy;
  decltype(&cublasLtMatmulDescCreate) desc_create;
  decltype(&cublasLtMatmulDescDestroy) desc_destroy;
  decltype(&cublasLtMatmulDescSetAttribute) desc_set;
  decltype(&cublasLtMatrixLayoutCreate) layout_create;
  decltype(&cublasLtMatrixLayoutDestroy) layout_destroy;
  decltype(&cublasLtMatmulPreferenceCreate) pref_create;
  decltype(&cublasLtMatmulPreferenceDestroy) pref_destroy;
  decltype(&cublasLtMatmulPreferenceSetAttribute) pref_set;
  decltype(&cublasLtMatmulAlgoGetHeuristic) heuristic;
  decltype(&cublasLtMatmul) matmul;
};


// Resolves the API once (thread-safe); R2M_ESTATE when cuBLASLt is missing.
int lt_api(LtApi **out);

}  // namespace r2m
