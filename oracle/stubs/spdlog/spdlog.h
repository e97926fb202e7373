/* No-op logging stand-in for the reference's logger macros (oracle recipe only). */
#ifndef VFB_ORACLE_STUB_SPDLOG_H
#define VFB_ORACLE_STUB_SPDLOG_H
namespace spdlog {
template <typename... A> inline void trace(A&&...) {}
template <typename... A> inline void debug(A&&...) {}
template <typename... A> inline void info(A&&...) {}
template <typename... A> inline void warn(A&&...) {}
template <typename... A> inline void error(A&&...) {}
template <typename... A> inline void critical(A&&...) {}
}
#endif
