// rsa_air.cuh — device side of the RSA-2048 AIR (layout and constraint order in rsa2048.hpp).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "rsa2048.hpp"

namespace sg {

// (n_records * 11041) x 32 column-major trace from the witnesses
// (d_rows: n_records * 32 rows, record-major).
cudaError_t rsa_expand(const rsa::RecordW* d_recs, const rsa::RowW* d_rows, uint64_t n_records, uint64_t* d_trace,
                       cudaStream_t s);
// Phi at the n_trace * blowup points of the LDE (record r's 11041 columns start at
// column r * 11041); d_part holds n_records * n values when n_records > 1.
cudaError_t rsa_phi(const uint64_t* d_lde, uint64_t n_records, uint64_t n_trace, uint64_t blowup, uint64_t* d_part,
                    uint64_t* d_phi, cudaStream_t s);

}  // namespace sg
