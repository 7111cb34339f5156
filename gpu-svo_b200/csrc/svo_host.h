// svo_host.h -- host-side pieces of the C ABI (mesh input, OBJ output).
#pragma once
#include <cstdint>

#include <nvtx3/nvToolsExt.h>

#include "svo_b200.h"

namespace svo::host {

void set_error(const char *msg);

// An NVTX range over a scope: the library's stages appear by name in Nsight
// Systems timelines (a no-op when no tool is attached).
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

// writeVoxel body (src/SVO.cu:755-777): one cube per surface voxel, origin =
// min + width * (x, y, z) computed on the host (separately rounded).
int write_voxels(const uint64_t *keys, int64_t n, const float origin[3], float width, const char *path);

// Installs a function a server calls, under its own lock, each time one of its
// requests finishes (built, failed or cancelled), with the request's ticket.
// The function must not call back into that server.  A fleet collects its
// members' completions this way.
void server_on_finish(svo_server *s, void (*fn)(void *arg, uint64_t ticket), void *arg);

}  // namespace svo::host
