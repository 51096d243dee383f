// metis_api.hpp -- the METIS 5.1 C entry points used for nested dissection.
//
// The engine links the METIS static library shipped with the CUDA toolkit, a
// 64-bit idx_t build.  Names, option indices and signatures follow the public
// METIS 5.1 manual.
#pragma once
#include <cstdint>

namespace cupf_b200 {
using idx_t = int64_t;
constexpr int METIS_NOPTIONS = 40;
constexpr int METIS_OK = 1;
constexpr int METIS_OPTION_SEED = 8;
constexpr int METIS_OPTION_NUMBERING = 17;
}  // namespace cupf_b200

extern "C" {
int METIS_SetDefaultOptions(cupf_b200::idx_t* options);
int METIS_NodeND(cupf_b200::idx_t* nvtxs, cupf_b200::idx_t* xadj, cupf_b200::idx_t* adjncy, cupf_b200::idx_t* vwgt,
                 cupf_b200::idx_t* options, cupf_b200::idx_t* perm, cupf_b200::idx_t* iperm);
int METIS_ComputeVertexSeparator(cupf_b200::idx_t* nvtxs, cupf_b200::idx_t* xadj, cupf_b200::idx_t* adjncy,
                                 cupf_b200::idx_t* vwgt, cupf_b200::idx_t* options, cupf_b200::idx_t* sepsize,
                                 cupf_b200::idx_t* part);
}
