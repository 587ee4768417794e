/* Extra forced include for Physics/SelfCollisionDetector.cpp only (test oracle).
   That file stores a pair hash into `c.hash`, a field SelfContact does not have
   (Physics/SelfCollisionDetector.cpp:566). After every standard header is in,
   `hash` is mapped onto Constraint::dLambda, an otherwise unused float, so the
   file compiles unchanged. */
#pragma once
#include "shim.h"
#include <unordered_map>
#include <unordered_set>
#include <string>
#include <iostream>
#define hash dLambda
