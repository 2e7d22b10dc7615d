// Large host blocks for the plan tables.  A process that builds plans again
// and again (a server: one hierarchy per request) would map fresh pages for
// every large table and take a page fault on the first touch of each, which
// costs about as much as filling the table.  Blocks of at least 1 MiB that
// are freed are kept here, up to a cap, and handed to later tables, so the
// pages are reused already mapped.  Smaller requests go to operator new.
#ifndef CMG_HOSTMEM_H
#define CMG_HOSTMEM_H

#include <cstddef>

namespace cmg {

// A block of at least `bytes` bytes (aligned for any type); throws
// std::bad_alloc.  A kept block is reused when it is at most twice the size
// asked for.
void* hostBlockAlloc(size_t bytes);
// Returns a block from hostBlockAlloc (`bytes` as asked for); it is kept for
// reuse while the kept bytes stay within hostBlockCap().
void hostBlockFree(void* p, size_t bytes);
// Bytes held for reuse, and the most that are held: min(8 GiB, physical
// memory / 8).
size_t hostBlockKept();
size_t hostBlockCap();
// Gives every kept block back to the system.
void hostBlockRelease();

}  // namespace cmg

#endif
