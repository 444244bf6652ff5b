// Shared host helpers of the C ABI (emp_common.h).
#include "emp_common.h"

namespace emp {

std::string& last_error()
{
    thread_local std::string message;
    return message;
}

void clear_error() { last_error().clear(); }

emp_status fail(emp_status status, const std::string& message)
{
    last_error() = message;
    return status;
}

emp_status cuda_fail(cudaError_t e, const char* what)
{
    const emp_status s = e == cudaErrorMemoryAllocation ? EMP_ERR_NOMEM : EMP_ERR_CUDA;
    cudaGetLastError();  // clear a sticky-free error so the next call starts clean
    return fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

emp_status select_device(int device, int* ordinal)
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(EMP_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
    if (device >= 0) {
        if (device >= count) return fail(EMP_ERR_INVALID, "device ordinal out of range");
        e = cudaSetDevice(device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
        *ordinal = device;
    } else {
        e = cudaGetDevice(ordinal);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    }
    return EMP_OK;
}

}  // namespace emp
