/*
 * cj_dlpack.h -- decoded images as DLPack tensors on the device.
 *
 * No counterpart in the reference: its output is copied to the host
 * (src/pixelTransformGPU.cu:664-669).  These entry points hand a decoded
 * image that is still in device memory to any framework that consumes
 * DLPack (torch.from_dlpack, cupy.from_dlpack, ...) without a copy.
 *
 * The structs below are the DLPack C ABI (the dlpack.h of the DLPack
 * project, v0.8 layout) declared here so that callers need no other header.
 */
#ifndef CJ_DLPACK_H
#define CJ_DLPACK_H

#include <stdint.h>

#include "cudajpeg.h"

#ifdef __cplusplus
extern "C" {
#endif

#ifndef DLPACK_VERSION
typedef enum { kDLCPU = 1, kDLCUDA = 2 } DLDeviceType;
typedef struct {
  DLDeviceType device_type;
  int32_t device_id;
} DLDevice;
typedef enum { kDLInt = 0U, kDLUInt = 1U, kDLFloat = 2U } DLDataTypeCode;
typedef struct {
  uint8_t code;
  uint8_t bits;
  uint16_t lanes;
} DLDataType;
typedef struct {
  void *data;
  DLDevice device;
  int32_t ndim;
  DLDataType dtype;
  int64_t *shape;
  int64_t *strides;
  uint64_t byte_offset;
} DLTensor;
typedef struct DLManagedTensor {
  DLTensor dl_tensor;
  void *manager_ctx;
  void (*deleter)(struct DLManagedTensor *self);
} DLManagedTensor;
#endif

/* Image i of the last run of batch b, in device memory, as a uint8 tensor:
 * [height, width, 3] (RGB), [height, width] (grey), or the flat
 * [bytes] buffer of the planar / NV12 formats.  NULL when image i was
 * rejected.  The tensor is a view of the batch's output buffer: it stays
 * valid until the batch is staged again or destroyed, and the work that
 * writes it is on the batch's stream (cjBatchStream).  The consumer calls
 * the tensor's deleter (or cjDLPackFree) when done; that frees only the
 * descriptor. */
DLManagedTensor *cjBatchDLPack(CJBatch *b, int i);

/* A finished server request's device pixels as a tensor shaped like
 * cjBatchDLPack's; valid until cjServerRelease(ticket).  NULL for an unknown,
 * unfinished or failed request. */
DLManagedTensor *cjServerDLPack(CJServer *s, long long ticket);

/* Calls t->deleter(t) (for callers that do not hand the tensor on). */
void cjDLPackFree(DLManagedTensor *t);

#ifdef __cplusplus
}
#endif
#endif /* CJ_DLPACK_H */
