// Forwards to the oracle's SZ3-ncp stand-in declarations.
#pragma once
#include "../../sz3_stub.hpp"
