// Error reporting shared by the translation units of libxpgi.so (defined in xpgi.cu; not exported).
#pragma once

#define XI_HIDDEN __attribute__((visibility("hidden")))

XI_HIDDEN int xi_fail(int code, const char* msg);      // records msg for xi_last_error, returns code
XI_HIDDEN int xi_cuda_check(const char* where);        // XI_E_CUDA with the pending CUDA error, else XI_OK
