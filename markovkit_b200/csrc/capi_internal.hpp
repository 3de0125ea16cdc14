// Internal to the C ABI: the handle types behind include/markovkit_b200.h and the mapping of
// C++ errors to MK_* status codes, shared by the translation units that implement entry points.
#pragma once

#include "../../include/markovkit_b200.h"
#include "assemble.hpp"
#include "engine.hpp"

#include <new>
#include <string>

struct mk_space_s {
    std::unique_ptr<mkb::Space> space;
};
struct mk_model_s {
    std::unique_ptr<mkb::Model> model;
};
struct mk_generator_s {
    std::unique_ptr<mkb::Space> space; // private copy of the geometry the generator indexes
    std::unique_ptr<mkb::Model> model; // private copy of the model (jumps on the host)
    std::unique_ptr<mkb::Generator> gen;
};
struct mk_csr_s {
    mkb::Csr csr;
};
struct mk_multigrid_s {
    std::unique_ptr<mkb::Multigrid> mg;
};
struct mk_precond_s {
    std::unique_ptr<mkb::Preconditioner> pc;
};
struct mk_solver_s {
    mk_generator gen = nullptr;
    mk_multigrid mg = nullptr;
    mk_precond pc = nullptr; // used when mg is null
    double shift = 0.0;
    mkb::GmresOptions opt;
    std::unique_ptr<mkb::Krylov> ws;
    mkb::DeviceArray<double> b, x; // staging for host-vector solves
};
struct mk_batch_solver_s {
    mk_generator gen = nullptr;
    mk_multigrid mg = nullptr;
    double shift = 0.0;
    mkb::GmresOptions opt;
    std::unique_ptr<mkb::KrylovBatch> ws;
    mkb::DeviceArray<double> b, x; // columns at the workspace's stride
};

namespace mkb::capi {

// the message of the calling thread's last failure (mk_last_error)
inline thread_local std::string g_last_error;

inline int fail(int code, const std::string &what) {
    g_last_error = what;
    return code;
}

template <typename F>
int guarded(F &&f) {
    try {
        f();
        return MK_OK;
    } catch (const Error &e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(MK_ENOMEM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(MK_EINVAL, e.what());
    }
}

inline cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }

// the right preconditioner of a resident solver, or null for plain GMRES
inline Preconditioner *preconditioner_of(const mk_solver_s &s) {
    if (s.mg) {
        return s.mg->mg.get();
    }
    return s.pc ? s.pc->pc.get() : nullptr;
}

} // namespace mkb::capi

#define MK_REQUIRE(cond, msg)                                                                      \
    do {                                                                                           \
        if (!(cond)) {                                                                             \
            throw ::mkb::Error(MK_EINVAL, msg);                                                    \
        }                                                                                          \
    } while (0)
