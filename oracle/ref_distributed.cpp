// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into or called by the
// product.  Only tests/ load the libraries this file is part of.
//
// The reference's distributed task table and coordinator checkpoint
// (src/distributed/task.cpp, src/distributed/checkpoint.cpp, compiled from
// the reference's sources by oracle/Makefile) behind a C interface, as the
// checker for wfpt.distributed: the same task list and task keys, and files
// each side writes that the other reads.
#include "distributed/checkpoint.hpp"
#include "distributed/task.hpp"

#include <cstdio>
#include <cstring>
#include <string>

extern "C" {

// createRenderTasks: up to `capacity` tasks as 7 uint32 each (tile ordinal,
// sample start, sample count, x, y, width, height); returns the task count.
uint64_t wfref_dist_tasks(uint32_t width, uint32_t height, uint32_t tile_width, uint32_t tile_height, uint32_t spp,
                          uint32_t spp_per_task, uint64_t fingerprint, uint32_t* out, uint64_t capacity) {
    std::vector<RenderTask> tasks =
        createRenderTasks(width, height, tile_width, tile_height, spp, spp_per_task, fingerprint);
    for (size_t i = 0; i < tasks.size() && i < capacity; ++i) {
        const RenderTask& t = tasks[i];
        uint32_t* o = out + 7 * i;
        o[0] = t.id.tileOrdinal;
        o[1] = t.id.sampleStart;
        o[2] = t.id.sampleCount;
        o[3] = t.tile.x;
        o[4] = t.tile.y;
        o[5] = t.tile.width;
        o[6] = t.tile.height;
    }
    return tasks.size();
}

uint64_t wfref_dist_task_key(uint64_t fingerprint, uint32_t tile, uint32_t sample_start, uint32_t sample_count) {
    return computeRenderTaskKey(fingerprint, RenderTaskId{tile, sample_start, sample_count});
}

// job: fingerprint, then width, height, tile width, tile height, spp, spp per task
int wfref_dist_checkpoint_write(const char* path, uint64_t fingerprint, const uint32_t* job, uint64_t sequence,
                                const float* radiance, const uint32_t* counts, const uint8_t* completed,
                                uint64_t task_count, char* error, uint64_t error_size) {
    DistributedCheckpoint c;
    c.job = DistributedJobConfig{fingerprint, job[0], job[1], job[2], job[3], job[4], job[5]};
    c.sequence = sequence;
    size_t pixels = size_t(job[0]) * job[1];
    c.accumulatedRadiance.resize(pixels);
    std::memcpy(c.accumulatedRadiance.data(), radiance, pixels * sizeof(DistributedRadiance));
    c.sampleCounts.assign(counts, counts + pixels);
    c.completedTasks.assign(completed, completed + task_count);
    std::string message;
    bool ok = writeDistributedCheckpoint(path, c, &message);
    if (!ok && error && error_size) std::snprintf(error, error_size, "%s", message.c_str());
    return ok ? 0 : 1;
}

// header: fingerprint, width, height, tile width, tile height, spp, spp per
// task, sequence, task count.  Payload arrays are filled when not NULL (they
// must hold width*height pixels and `task count` flags).  0 on success.
int wfref_dist_checkpoint_read(const char* path, uint64_t* header, float* radiance, uint32_t* counts,
                               uint8_t* completed, char* error, uint64_t error_size) {
    DistributedCheckpoint c;
    std::string message;
    if (!readDistributedCheckpoint(path, c, &message)) {
        if (error && error_size) std::snprintf(error, error_size, "%s", message.c_str());
        return 1;
    }
    header[0] = c.job.jobFingerprint;
    header[1] = c.job.width;
    header[2] = c.job.height;
    header[3] = c.job.tileWidth;
    header[4] = c.job.tileHeight;
    header[5] = c.job.samplesPerPixel;
    header[6] = c.job.samplesPerTask;
    header[7] = c.sequence;
    header[8] = c.completedTasks.size();
    if (radiance) std::memcpy(radiance, c.accumulatedRadiance.data(), c.accumulatedRadiance.size() * 12);
    if (counts) std::memcpy(counts, c.sampleCounts.data(), c.sampleCounts.size() * 4);
    if (completed) std::memcpy(completed, c.completedTasks.data(), c.completedTasks.size());
    return 0;
}

}  // extern "C"
