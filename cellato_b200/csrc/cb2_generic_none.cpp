// cb2_generic_none.cpp -- stands in for cb2_generic.cu when the library is
// built without the Cellato headers: no lowered DSL automata are registered,
// and the hand-written networks (ids 0-2) are all the library runs.
#include <vector>

#include "cb2_batch.h"
#include "cb2_internal.h"

namespace cb2 {

int generic_count() { return 0; }

uint64_t builtin_fingerprint(int) { return 0; }

const automaton_desc* generic_desc(int) { return nullptr; }

const std::vector<strip_variant>& generic_variants(int) {
    static const std::vector<strip_variant> none;
    return none;
}

const void* generic_batch_kernel() { return nullptr; }

} // namespace cb2
