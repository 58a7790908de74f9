// dump.h -- asynchronous trajectory writer of an engine (the reference's all.trj,
// src/system/dump.cu:23-201).  A frame is a device-side snapshot of replica 0's slots
// (taken on the engine stream when its step ends), copied to pinned host memory on a
// copy stream and converted, formatted and written by a host thread while the device
// keeps stepping.  Two snapshot slots: a third frame waits for the older one's write.
#pragma once
#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdio>
#include <deque>
#include <mutex>
#include <string>
#include <thread>

#include "dpd_common.h"

namespace dpd {

struct DumpWriter {
    std::string path;
    std::string id;                    // "" for the dump command, else the compute's ID
    FILE* file = nullptr;
    uint32_t start = 0, every = 1;
    bool unwrapped = false, force = false, vel = false;
    uint32_t group = 0;                // compute dump: the group's types (0 = every atom)
    bool mol = false;                  // compute dump of a molecular system: id mol type x y z
    int ns = 0;                        // slots of replica 0 (a multiple of 32)
    float4 *dpos[2] = {}, *dvel[2] = {}, *dfrc[2] = {};
    int4* dimg[2] = {};
    FixOut* dfo[2] = {};
    float4 *hpos[2] = {}, *hvel[2] = {}, *hfrc[2] = {};
    int4* himg[2] = {};
    FixOut* hfo[2] = {};
    cudaStream_t copy = nullptr;
    cudaEvent_t taken[2] = {}, copied[2] = {};
    uint32_t step[2] = {0, 0};
    bool busy[2] = {false, false};
    int next_slot = 0;
    int64_t frames = 0;
    std::deque<int> queue;             // slots waiting for the writer
    bool stop = false;
    std::string error;                 // first write or copy error
    std::mutex mu;
    std::condition_variable cv;
    std::thread thread;
};

}  // namespace dpd
