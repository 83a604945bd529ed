// verifier.hpp — host STIR verifier entry (see verifier.cpp).
#pragma once
#include "protocol.hpp"

namespace sg {
bool stir_verify(const StirProof& pr, const sg_fri_params& p);
}
