// The reference formats with fmt; the header-only copy bundled with spdlog serves (FMT_HEADER_ONLY).
#pragma once
#include <spdlog/fmt/bundled/format.h>
