// Link-only test doubles for src/25DCannonNCCL.cpp, which the oracle compiles for its
// truncatedDivisionRemainer (25DCannonNCCL.cpp:6-9) and the decomposer's overlap hook.
// The oracle runs only the MPI step loop (src/25DCannon.cpp:286-375); any NCCL call
// aborts the in-process job instead of pretending to communicate.
#include <cuda_runtime.h>
#include <nccl.h>

#include "mpi.h"

static ncclResult_t refuse() {
    MPI_Abort(MPI_COMM_WORLD, -77);
    return ncclInvalidUsage;
}

extern "C" {
ncclResult_t ncclGetUniqueId(ncclUniqueId*) { return refuse(); }
ncclResult_t ncclCommInitRank(ncclComm_t*, int, ncclUniqueId, int) { return refuse(); }
ncclResult_t ncclCommSplit(ncclComm_t, int, int, ncclComm_t*, ncclConfig_t*) { return refuse(); }
const char* ncclGetErrorString(ncclResult_t) { return "NCCL is not available in the oracle"; }
ncclResult_t ncclReduce(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, int, ncclComm_t, cudaStream_t) {
    return refuse();
}
ncclResult_t ncclBroadcast(const void*, void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) {
    return refuse();
}
ncclResult_t ncclSend(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) { return refuse(); }
ncclResult_t ncclRecv(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) { return refuse(); }
ncclResult_t ncclGroupStart() { return refuse(); }
ncclResult_t ncclGroupEnd() { return refuse(); }

cudaError_t cudaStreamCreate(cudaStream_t* s) {
    *s = nullptr;
    return cudaSuccess;
}
cudaError_t cudaStreamWaitEvent(cudaStream_t, cudaEvent_t, unsigned int) { return cudaSuccess; }
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
cudaError_t cudaEventCreate(cudaEvent_t* e) {
    *e = nullptr;
    return cudaSuccess;
}
cudaError_t cudaEventRecord(cudaEvent_t, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaMallocAsync(void** p, size_t n, cudaStream_t) { return cudaMalloc(p, n); }
}
