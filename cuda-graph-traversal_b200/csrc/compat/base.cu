// base.cu -- the arena of the reference's src/base.h (src/base.cu:5-78):
// a bump allocator over one host malloc or one device allocation.
#include "base.h"

u64 mem_align_forward(u64 size, u64 alignment) { return (size + alignment - 1) & ~(alignment - 1); }

void *_arena_push(Arena *arena, u64 size, u64 alignment) {
    if (!arena->base) {
        ERROR("Arena was not initialized");
        return 0;
    }
    const u64 start = mem_align_forward(arena->used, alignment);
    if (start + size > arena->reserved) {
        ERROR("Arena out of space");
        return 0;
    }
    arena->used = start + size;
    return (u8 *)arena->base + start;
}

Arena arena_create_cpu(u64 capacity) {
    Arena a;
    a.reserved = mem_align_forward(capacity, ARENA_DEFAULT_ALIGNMENT);
    a.used = 0;
    a.base = malloc(a.reserved);
    return a;
}

Arena arena_create_gpu(u64 capacity) {
    Arena a;
    a.reserved = mem_align_forward(capacity, ARENA_DEFAULT_ALIGNMENT);
    a.used = 0;
    a.base = 0;
    if (a.reserved && cudaMalloc(&a.base, a.reserved) != cudaSuccess) {
        ERROR("Failed to allocate GPU arena of %llu bytes", (unsigned long long)a.reserved);
        ABORT();
    }
    return a;
}

Arena arena_from_arena(Arena *arena, u64 capacity) {
    Arena a;
    a.reserved = mem_align_forward(capacity, ARENA_DEFAULT_ALIGNMENT);
    a.used = 0;
    a.base = arena_push(arena, a.reserved);
    return a;
}

void arena_release_cpu(Arena *arena) {
    if (!arena->base) return;
    free(arena->base);
    arena->reserved = arena->used = 0;
    arena->base = 0;
}

void arena_release_gpu(Arena *arena) {
    if (!arena->base) return;
    cudaFree(arena->base);
    arena->reserved = arena->used = 0;
    arena->base = 0;
}

void arena_clear(Arena *arena) { arena->used = 0; }
