/*
 * Zero-filling global allocation for the oracle build of the reference.
 *
 * The reference leaves several arrays uninitialised and then reads them:
 * the TDBC state Psi (calculation_2D.cpp:128-134, read by Cal_TDBC at
 * :1019-1028 before its first update), the "nn" field buffers whose
 * boundary nodes are read by the BC sweeps before any write, and object
 * members that only some branches set. Zero-filling every allocation makes
 * the reference deterministic; the B200 implementation starts from the
 * same zero state. Test infrastructure only.
 */
#include <cstdlib>
#include <new>

static void *oracle_zalloc(std::size_t n)
{
    void *p = std::calloc(n ? n : 1, 1);
    if (!p) throw std::bad_alloc();
    return p;
}

void *operator new(std::size_t n) { return oracle_zalloc(n); }
void *operator new[](std::size_t n) { return oracle_zalloc(n); }
void operator delete(void *p) noexcept { std::free(p); }
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete(void *p, std::size_t) noexcept { std::free(p); }
void operator delete[](void *p, std::size_t) noexcept { std::free(p); }
