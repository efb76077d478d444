// Helpers shared by the C-ABI translation units.
#pragma once

#include <string>

#include "../../include/phmm_b200.h"

namespace phmm {

class Engine;

phmm_status set_error(phmm_status st, const std::string& msg);
void clear_error();
Engine* engine_of(phmm_engine* e);
// Stops and frees the serving loop attached to an engine, if any (phmm_serve.cpp).
void server_release(phmm_engine* e);

}  // namespace phmm
