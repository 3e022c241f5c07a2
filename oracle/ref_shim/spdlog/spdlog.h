// Stand-in for spdlog (TEST INFRASTRUCTURE for oracle/_ref): the reference
// uses it only for log lines, which the harness discards.
#pragma once
#include <string>

#define SPDLOG_LEVEL_TRACE 0
#define SPDLOG_LEVEL_DEBUG 1
#define SPDLOG_LEVEL_INFO 2
#define SPDLOG_LEVEL_WARN 3
#define SPDLOG_LEVEL_ERROR 4
#define SPDLOG_LEVEL_CRITICAL 5
#define SPDLOG_LEVEL_OFF 6
#ifndef SPDLOG_ACTIVE_LEVEL
#define SPDLOG_ACTIVE_LEVEL SPDLOG_LEVEL_OFF
#endif
#define SPDLOG_TRACE(...) (void)0
#define SPDLOG_DEBUG(...) (void)0
#define SPDLOG_INFO(...) (void)0
#define SPDLOG_WARN(...) (void)0
#define SPDLOG_ERROR(...) (void)0
#define SPDLOG_CRITICAL(...) (void)0

namespace spdlog {
namespace level {
enum level_enum { trace, debug, info, warn, err, critical, off };
}
inline void set_pattern(const std::string&) {}
inline void set_level(level::level_enum) {}
}  // namespace spdlog
