// Test-infrastructure shim for building the reference T-BLAEQ sources without cuVS.
//
// The reference selects its GPU k-means backend through src/Kmeans/CUDAKmeans.cuh
// (cuVS, src/Kmeans/CUDAKmeans.cu:65-97). cuVS is not installed in this image, so the
// oracle build puts this directory ahead of the reference root on the include path and
// aliases the GPU backend to the reference's own header-only CPU Lloyd implementation
// (src/Kmeans/CPUKmeans.cuh). The query path and the synthetic RandomKmeans generator do
// not use k-means at all, so both are unaffected.
#pragma once
#include "src/Kmeans/CPUKmeans.cuh"
using CUDAKmeans = CPUKmeans;
