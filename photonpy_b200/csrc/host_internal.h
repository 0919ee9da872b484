// Host-side services of estimator.cu shared with the other host translation units.
#pragma once
#include <cstddef>
#include <string>

struct Context;

namespace pb200 {

// Registers a non-estimator object with a context: Context_Destroy calls destroy(obj) for each
// registered object (before it deletes the context's estimators). detach is a no-op when the
// object is not registered.
void context_attach(Context* ctx, void* obj, void (*destroy)(void*));
void context_detach(Context* ctx, void* obj);

// Pinned host blocks from a process-wide cache (blocks of deleted queues are kept for the next
// one, up to 2 GB). give() takes back exactly what take() handed out.
void* pinned_take(size_t bytes);
void pinned_give(void* p, size_t bytes);

// Records `msg` as this thread's last error (PB200_GetLastError) and prints it through the
// debug-print callback.
void set_last_error(const std::string& msg);

}  // namespace pb200
