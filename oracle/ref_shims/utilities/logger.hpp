// Stand-in for the rapids-logger based logging macros (force-included): no-ops.
#pragma once
#define CUOPT_LOG_TRACE(...) \
  do {                       \
  } while (0)
#define CUOPT_LOG_DEBUG(...) \
  do {                       \
  } while (0)
#define CUOPT_LOG_INFO(...) \
  do {                      \
  } while (0)
#define CUOPT_LOG_WARN(...) \
  do {                      \
  } while (0)
#define CUOPT_LOG_ERROR(...) \
  do {                       \
  } while (0)
