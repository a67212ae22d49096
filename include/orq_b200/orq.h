// orq.h — the loopback build of ORQ's user API on one B200.
//
// A program written against ORQ's orq.h (include/orq.h and the type macros
// of include/mpc.h:70-169) compiles against this header: with `-I
// include/orq_b200` the same
//
//     #include "orq.h"
//     using namespace orq::service;
//     using namespace COMPILED_MPC_PROTOCOL_NAMESPACE;
//     int main(int argc, char** argv) { orq_init(argc, argv); ... }
//
// gets BSharedVector<T> / ASharedVector<T> with their operators,
// secret_share_b / secret_share_a / public_share / secret_share,
// orq::operators (sorts, shuffle, permutations, compare_rows, swap,
// multiplex, table_sort, distinct), orq::aggregators and EncodedTable<T> with
// sort / aggregate / joins / open_with_schema. One process plays all the
// parties (replicated 3PC, or 2PC / 4PC with -DPROTOCOL_NUM=2|4); every
// protocol step runs in liborq_cuda.so (link
// with -L<dir> -lorq_cuda) through the C ABI of orq_cuda.h. With the same
// keys and one worker thread at batch size -1 on the CPU side, shares equal a
// CPU run's bit for bit.
#pragma once

#include <iostream>

#include "encoded_table.hpp"
#include "operators.hpp"
#include "runtime.hpp"
#include "shared_vector.hpp"

namespace orq {
namespace debug {
// single_cout of the reference's debug helpers: every party prints, and here
// there is one process
#define single_cout(x) (std::cout << x << std::endl)
#define single_cout_nonl(x) (std::cout << x)
}  // namespace debug

namespace service {
namespace loopback {
template <typename T>
using BSharedVector = orq::BSharedVector<T>;
template <typename T>
using ASharedVector = orq::ASharedVector<T>;
template <typename T>
using EncodedTable = orq::relational::EncodedTable<T>;
template <typename T>
using Vector = orq::Vector<T>;
template <typename T>
using DataTable = orq::DataTable<T>;
using EncodedColumn = orq::relational::EncodedColumn;
using orq::public_share;
using orq::secret_share_a;
using orq::secret_share_b;
using orq::secret_share_vec;
using orq::relational::secret_share;
using namespace orq::aggregators;
using orq::relational::AggregationOptions;
using orq::relational::ENC_TABLE_JOIN_ID;
using orq::relational::ENC_TABLE_VALID;
using orq::relational::isBShared;
using orq::relational::JoinOptions;
using orq::operators::ASC;
using orq::operators::DESC;
}  // namespace loopback
// the protocol namespaces of mpc.h: one loopback API serves all three
namespace loopback_3pc = loopback;
namespace loopback_2pc = loopback;
namespace loopback_4pc = loopback;
}  // namespace service
}  // namespace orq

// PROTOCOL_NUM (mpc.h:70-169) picks the protocol at compile time, as in the
// reference: 3 replicated 3PC (default), 2 Beaver 2PC with dummy triples, 4
// Fantastic-4PC. The 2PC / 4PC runtimes run sharing, open, and_b, xor_b,
// multiply_a, add_a, sub_a and b2a_bit; other operators throw RuntimeError.
#ifndef PROTOCOL_NUM
#define PROTOCOL_NUM 3
#endif
#if PROTOCOL_NUM == 2
#define COMPILED_MPC_PROTOCOL_NAMESPACE orq::service::loopback_2pc
#elif PROTOCOL_NUM == 4
#define COMPILED_MPC_PROTOCOL_NAMESPACE orq::service::loopback_4pc
#elif PROTOCOL_NUM == 3
#define COMPILED_MPC_PROTOCOL_NAMESPACE orq::service::loopback_3pc
#else
#error "PROTOCOL_NUM must be 2, 3 or 4"
#endif

// orq_init (include/backend/common/setup.h:8-58): the reference reads the
// party/thread/batch arguments and connects the parties; the loopback build
// creates the one runtime that plays all parties. The PRG keys come from
// ORQ_SEED (default 1) exactly as the deterministic key generator of the
// reference's test build derives them; ORQ_DEVICE picks the CUDA device.
inline void orq_init(uint64_t seed, int device = 0) {
    orq::service::runtime_holder() = std::make_unique<orq::service::LoopbackRunTime>(seed, device, PROTOCOL_NUM);
}
inline void orq_init(int argc = 0, char** argv = nullptr) {
    (void)argc;
    (void)argv;
    const char* s = std::getenv("ORQ_SEED");
    const char* d = std::getenv("ORQ_DEVICE");
    orq_init(s ? std::strtoull(s, nullptr, 10) : 1ull, d ? std::atoi(d) : 0);
}
// tears the runtime down (the reference's parties exit with the process)
inline void orq_finalize() { orq::service::runtime_holder().reset(); }
