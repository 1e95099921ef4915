// Library-internal interface of the packed batch engine (sdr_gpu.cu), used
// by the batch and serving layer (serving.cpp). Not part of the C ABI.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "sdr_gpu.h"

struct PackedEngine;

// A scene that left the engine: finished (status SDR_OK, with its summary
// and stats) or failed.
struct PackedDone {
    uint64_t tag = 0;
    int32_t status = SDR_OK;
    std::string error;
    sdr_summary summary{};
    sdr_solver_stats stats{};
};

// nullptr on failure (message through sdr_last_error).
PackedEngine* packed_engine_create(int32_t device);
// Creates the scene's solver (particle capacity `capacity`) on the engine's
// stream; a scene that cannot start is reported in `done` at once.
int packed_engine_add(PackedEngine* e, const sdr_scene_desc& d, uint64_t capacity, uint64_t tag,
                      std::vector<PackedDone>& done);
size_t packed_engine_live(const PackedEngine* e);
// One substep of every live scene, one launch per substep operation for all of
// them; scenes that completed their last frame (or failed) go to `done`.
void packed_engine_step(PackedEngine* e, std::vector<PackedDone>& done);
// Launches, packed steps, graph captures and the autotuned CTAs per SM (0
// while still tuning).
void packed_engine_counters(const PackedEngine* e, uint64_t* launches, uint64_t* steps, uint64_t* captures,
                            int* ctas_per_sm);
void packed_engine_destroy(PackedEngine* e);
