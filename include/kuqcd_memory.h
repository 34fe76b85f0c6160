/*
 * Host storage of the class-level API (the reference's kuqcd_memory.h:25-84): KMemory owns the bytes of a field,
 * Index an integer table.  Field storage is page-locked host memory from libkuqcd_b200 (kq_host_alloc), so that the
 * copies to and from the GPU that every field operation makes run at full link speed; it falls back to plain
 * 64-byte aligned memory, as the reference allocates, when page-locking is refused.
 */
#ifndef KUQCD_MEMORY_H
#define KUQCD_MEMORY_H

#include <cstdlib>
#include <cstring>
#include <new>

#include "kuqcd_b200.h"
#include "kuqcd_utils.h"

namespace kuqcd {

class KMemory {
public:
    size_t size = 0;
    void *rawPtr = nullptr;

    KMemory() = default;
    explicit KMemory(size_t sz) { InitMem(sz); }
    KMemory(const KMemory &mem)
    {
        InitMem(mem.size);
        Copy(mem);
    }
    KMemory &operator=(const KMemory &mem)
    {
        if (this != &mem) {
            if (size != mem.size) {
                Free();
                InitMem(mem.size);
            }
            Copy(mem);
        }
        return *this;
    }
    void InitMem(size_t sz)
    {
        if (!Alloc(sz)) throw std::bad_alloc();
    }
    virtual bool Alloc(size_t sz)
    {
        Free();
        void *p = nullptr;
        if (kq_host_alloc(sz, &p) != KUQCD_SUCCESS) return false;
        rawPtr = p;
        size = sz;
        return true;
    }
    void Copy(const KMemory &mem)
    {
        if (rawPtr && mem.rawPtr) std::memcpy(rawPtr, mem.rawPtr, size < mem.size ? size : mem.size);
    }
    void Clear()
    {
        if (rawPtr) std::memset(rawPtr, 0, size);
    }
    virtual void Free()
    {
        if (rawPtr) kq_host_free(rawPtr);
        rawPtr = nullptr;
        size = 0;
    }
    virtual ~KMemory() { Free(); }
};

class Index {
public:
    size_t length = 0;
    long *idx = nullptr;

    Index() = default;
    explicit Index(size_t len) { Init(len); }
    Index(const Index &other) { *this = other; }
    Index &operator=(const Index &other)
    {
        if (this != &other) {
            Init(other.length);
            if (other.length) std::memcpy(idx, other.idx, other.length * sizeof(long));
        }
        return *this;
    }
    void Init(size_t len)
    {
        if (!Alloc(len)) throw std::bad_alloc();
    }
    bool Alloc(size_t len)
    {
        Free();
        if (len == 0) return true;
        idx = static_cast<long *>(std::malloc(len * sizeof(long)));
        if (!idx) return false;
        length = len;
        return true;
    }
    void Free()
    {
        std::free(idx);
        idx = nullptr;
        length = 0;
    }
    ~Index() { Free(); }
};

}  // namespace kuqcd

#endif
