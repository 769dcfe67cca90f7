// The reference's debug printing reaches fmt through DARMA/vt's transport header; for the single-rank host
// cross-check fmt alone serves.
#pragma once
#include <fmt/format.h>
