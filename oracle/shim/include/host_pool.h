/*
 * Host memory behind the test doubles' cudaMalloc (fake_cuda.cpp) and the in-process
 * MPI's message buffers (fake_mpi.cpp), and the copies the doubles make.  Freed blocks are kept and handed out again by
 * size, so the reference's driver, which allocates its tiles and messages afresh on every
 * call, does not pay the kernel's first-touch page faults on every call: a real cudaMalloc
 * returns device memory that is already mapped, and a real MPI keeps its buffers.  Test
 * infrastructure only.
 */
#ifndef ORACLE_HOST_POOL_H
#define ORACLE_HOST_POOL_H
#include <cstddef>

void* host_pool_alloc(size_t bytes);  // uninitialised, 64-byte aligned; nullptr when out of memory
void host_pool_free(void* p);         // p from host_pool_alloc (or nullptr)

// memmove / memset that split large transfers across the process's host cores, as a copy
// engine moves a device buffer at memory bandwidth rather than at one core's memcpy rate.
void host_copy(void* dst, const void* src, size_t bytes);
void host_zero(void* dst, size_t bytes);

// Owning byte buffer from the pool (movable, not copyable).
struct PoolBytes {
    unsigned char* p = nullptr;
    size_t n = 0;
    PoolBytes() = default;
    explicit PoolBytes(size_t bytes) : p(static_cast<unsigned char*>(host_pool_alloc(bytes ? bytes : 1))), n(bytes) {}
    PoolBytes(PoolBytes&& o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    PoolBytes& operator=(PoolBytes&& o) noexcept {
        if (this != &o) {
            host_pool_free(p);
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    PoolBytes(const PoolBytes&) = delete;
    PoolBytes& operator=(const PoolBytes&) = delete;
    ~PoolBytes() { host_pool_free(p); }
    unsigned char* data() { return p; }
    const unsigned char* data() const { return p; }
    size_t size() const { return n; }
};
#endif
