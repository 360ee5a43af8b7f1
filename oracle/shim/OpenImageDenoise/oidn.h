/* Declarations that let the reference's data/include/data/denoise.h compile
 * without OpenImageDenoise (not installed here). The reference CUDA harness
 * never constructs a TransferStream or OIDNDenoiser, so none of these
 * functions is called or linked; the denoise stage is not part of the traced
 * path and is not built. */
#pragma once
#include <cstddef>
#include <cuda_runtime.h>
typedef struct OIDNDeviceImpl* OIDNDevice;
typedef struct OIDNFilterImpl* OIDNFilter;
typedef enum { OIDN_QUALITY_DEFAULT = 0, OIDN_QUALITY_FAST = 4, OIDN_QUALITY_BALANCED = 5,
               OIDN_QUALITY_HIGH = 6 } OIDNQuality;
typedef enum { OIDN_FORMAT_FLOAT3 = 3 } OIDNFormat;
typedef enum { OIDN_ERROR_NONE = 0 } OIDNError;
OIDNDevice oidnNewCUDADevice(const int*, const cudaStream_t*, int);
void oidnCommitDevice(OIDNDevice);
OIDNFilter oidnNewFilter(OIDNDevice, const char*);
void oidnSetSharedFilterImage(OIDNFilter, const char*, void*, OIDNFormat, size_t, size_t, size_t, size_t, size_t);
void oidnSetFilterBool(OIDNFilter, const char*, bool);
void oidnSetFilterInt(OIDNFilter, const char*, int);
void oidnSetFilterFloat(OIDNFilter, const char*, float);
void oidnCommitFilter(OIDNFilter);
void oidnExecuteFilterAsync(OIDNFilter);
OIDNError oidnGetDeviceError(OIDNDevice, const char**);
void oidnReleaseFilter(OIDNFilter);
void oidnReleaseDevice(OIDNDevice);
