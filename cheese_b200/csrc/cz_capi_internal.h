// The C ABI's handle types (shared by the translation units that implement include/cheese_b200.h).
#pragma once
#include "../../include/cheese_b200.h"
#include "cz_clifford.h"
#include "cz_engine.h"
#include "cz_rus.h"
#include "cz_spec.h"
#include "cz_tcount.h"

#include <string>

struct cz_spec { cz::HostSpec hs; };
struct cz_batch { cz::BatchSession *b; std::string err; };
struct cz_engine { cz::Engine *e; cz::TcountContext *tc; cz::CliffordContext *cl; cz::RusContext *ru; };
