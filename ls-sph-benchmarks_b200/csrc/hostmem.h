// hostmem.h -- which page-locked host buffers a kernel may access in place.
//
// lssph_upload / lssph_download move the particle state with one kernel when every field
// buffer is page-locked and mapped into the device's address space (what cudaHostAlloc and
// torch's pin_memory return).  A kernel may load from any such buffer, but it may store
// only into one the device can write: memory registered with cudaHostRegisterReadOnly is
// mapped too, yet a store into it is an invalid access.  The flags are the access flags
// cuPointerGetAttribute(CU_POINTER_ATTRIBUTE_ACCESS_FLAGS) reports for the current device
// (0 none, 1 read, 3 read-write), or -1 when the driver could not be asked.  Buffers that
// fail the test go through cudaMemcpyAsync instead, which reports errors on the host.
#ifndef LSSPH_HOSTMEM_H
#define LSSPH_HOSTMEM_H

namespace lssph {

constexpr long long kAccessRead = 0x1;        // CU_POINTER_ATTRIBUTE_ACCESS_FLAG_READ
constexpr long long kAccessReadWrite = 0x3;   // CU_POINTER_ATTRIBUTE_ACCESS_FLAG_READWRITE

inline bool mapped_store_allowed(long long flags) { return flags == kAccessReadWrite; }

}  // namespace lssph

#endif
