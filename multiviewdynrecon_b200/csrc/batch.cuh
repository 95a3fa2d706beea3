// Host-side state of the solver shared by the C ABI files: the batch object
// (a single solver is a batch of one) and the input binding.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "mvdr_internal.cuh"

namespace mvdr {

// solver-owned device copies of inputs (mvdr_set_inputs_host,
// mvdr_set_inputs_textures)
struct OwnedInputs {
    void* mem = nullptr;
    size_t bytes = 0;
};

struct Batch {
    mvdr_config cfg{};
    LaunchCfg lc{};
    uint32_t B = 0;
    uint32_t cap_edges = 0;
    std::vector<InstDesc> host;
    InstDesc* d_inst = nullptr;
    uint32_t* d_bars = nullptr;  // persistent PCG barrier counters
    // the stream beside the solve's stream and the events that fork it from
    // and join it back (launch_assemble_forked)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    size_t per_inst_bytes = 0;
    std::vector<OwnedInputs> owned;   // host-input copies per instance
    std::vector<OwnedInputs> staged;  // texture-map copies per instance
    std::vector<mvdr_inputs> bound;   // the inputs last bound per instance (device pointers)
    std::vector<uint8_t> has_inputs;
    // the descriptor last copied to d_inst per instance: a rebind with the
    // same buffers and sizes skips the (pageable, possibly blocking) upload
    std::vector<InstDesc> uploaded;
    std::vector<uint8_t> uploaded_valid;
    uint32_t gn_iter = 0;
    // graph cache: (gn, pcg) -> exec
    std::map<std::pair<uint32_t, uint32_t>, cudaGraphExec_t> graphs;
    std::vector<struct SolverView*> views;

    ~Batch();
};

// record `msg` as the last error of this host thread; returns `code`
int fail(int code, const std::string& msg);
// validate *in against the batch's capacities
int check_inputs(const Batch& b, const mvdr_inputs* in);
// bind device-pointer inputs to instance `inst` and reset its warp field
int bind_inputs(Batch& b, uint32_t inst, const mvdr_inputs* in, cudaStream_t st);

}  // namespace mvdr

struct mvdr_solver {
    mvdr::Batch* batch;
    uint32_t inst;
    bool owns;
};
struct mvdr_batch {
    mvdr::Batch* batch;
};

namespace mvdr {

struct SolverView {
    mvdr_solver s;
};

}  // namespace mvdr
