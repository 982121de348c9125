// nccl_dl.hpp — NCCL resolved at run time with dlopen.  A process that already holds libnccl.so.2
// reuses that copy; otherwise the library named by PHX_NCCL_LIB, else the system one, is loaded.
// Linking libphx.so against one NCCL would let two libraries of the same soname meet in one process
// (a framework loaded later would then find an older NCCL than the one it was built against).
#pragma once

#include <nccl.h>

#include <string>

namespace phx {

struct NcclApi {
    ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*AllGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Broadcast)(const void *, void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

// The loaded API, or nullptr with a reason in *why.
const NcclApi *nccl_api(std::string *why);

} // namespace phx
