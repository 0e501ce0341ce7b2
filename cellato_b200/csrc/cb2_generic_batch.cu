// cb2_generic_batch.cu -- the batch kernel over every registered automaton:
// the hand-written networks and the lowered DSL rules of cb2_dsl_configs.h
// (ids kNumBuiltin.. in list order).  A batch holding a lowered rule runs
// this kernel (kind kBatchAll); its tasks pass each chunk's first
// generation, the grid's rows and its seed to the window rules, so
// stochastic, Margolus and alternating rules advance exactly as in the strip
// kernels.  The lowered rules pass two rows per barrier, as their strip
// plans do: their windows hold 3P words per row and level.
//
// Built only when the Cellato headers are present; cb2_generic_none.cpp
// stands in otherwise and reports no kernel.
// The batch kernels keep plain copies of the planes a rule passes on (cb2_rules.cuh fresh).
#define CB2_PLAIN_COPIES
#include <cuda_runtime.h>

#include <type_traits>

#include "cb2_ast.cuh"
#include "cb2_batch_kernel.cuh"
#include "cb2_dsl_configs.h"
#include "cb2_internal.h"
#include "cb2_rules.cuh"

namespace cb2 {
namespace {

constexpr int kNetRows = 4;  // the hand-written networks, as in their own batch kernel
constexpr int kDslRows = 2;
constexpr int kWarps = kBatchKindWarps[kBatchAll];
constexpr int kSmem = batch_smem_words(kMaxPlanes, kDslRows, kWarps);
static_assert(batch_smem_words(3, kNetRows, kWarps) <= kSmem, "network pipelines larger than the lowered rules'");

template <class... C>
struct config_list {};
struct list_end {};

// Lowered rule number I, I+1, ... of the list: the one whose id is `id`.
template <int I, class C, class... Rest>
__device__ __forceinline__ void run_lowered(int id, int k, const strip_task& t, const lane_geom<1>& geom,
                                            uint32_t* smem) {
    if constexpr (!std::is_same_v<C, list_end>) {
        if (id == I)
            batch_run_rule<ast_rule<C>, kBatchKMax, kDslRows, kSmem, kWarps>(t, k, geom, smem);
        else
            run_lowered<I + 1, Rest...>(id, k, t, geom, smem);
    }
}

template <class L>
struct lowered;
template <class... C>
struct lowered<config_list<C...>> {
    __device__ __forceinline__ static void run(int id, int k, const strip_task& t, const lane_geom<1>& geom,
                                               uint32_t* smem) {
        run_lowered<kNumBuiltin, C...>(id, k, t, geom, smem);
    }
};

#define CB2_CONFIG_TYPE(C, NAME) C,
#define CB2_USER_TYPE(C) C,
#ifdef CB2_USER_CONFIGS
using all_configs = config_list<CB2_DSL_CONFIGS(CB2_CONFIG_TYPE) CB2_USER_CONFIGS(CB2_USER_TYPE) list_end>;
#else
using all_configs = config_list<CB2_DSL_CONFIGS(CB2_CONFIG_TYPE) list_end>;
#endif
#undef CB2_CONFIG_TYPE
#undef CB2_USER_TYPE

struct all_rules {
    static constexpr int kWarps = cb2::kWarps;
    static constexpr int kSmemWords = kSmem;
    static constexpr bool kTimed = true;
    __device__ __forceinline__ static void run(int automaton, int k, const strip_task& t, const lane_geom<1>& geom,
                                               uint32_t* smem) {
        switch (automaton) {
        case 0: batch_run_rule<game_of_life, kBatchKMax, kNetRows, kSmem, kWarps>(t, k, geom, smem); break;
        case 1: batch_run_rule<wire, kBatchKMax, kNetRows, kSmem, kWarps>(t, k, geom, smem); break;
        case 2: batch_run_rule<excitable, kBatchKMax, kNetRows, kSmem, kWarps>(t, k, geom, smem); break;
        default: lowered<all_configs>::run(automaton, k, t, geom, smem); break;
        }
    }
};

} // namespace

const void* generic_batch_kernel() { return (const void*)batch_kernel<all_rules>; }

} // namespace cb2
