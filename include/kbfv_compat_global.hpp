// kbfv_compat_global.hpp -- the compat classes of kbfv_compat.hpp under the
// unqualified names the reference's drivers use (kunpBFV declares its classes
// in the global namespace, include/BFVcontext.h:17, include/BFVScheme.h:12,
// include/Plaintext.cuh:6, include/Ciphertext.cuh:5, include/SecretKey.cuh:10;
// uint64_tt in include/uint128.cuh:15). Included by the forwarding headers of
// include/kunpbfv/include/.
#pragma once

#include "kbfv_compat.hpp"

using kbfv_compat::BFVContext;
using kbfv_compat::BFVScheme;
using kbfv_compat::Ciphertext;
using kbfv_compat::Plaintext;
using kbfv_compat::SecretKey;
using kbfv_compat::uint64_tt;
