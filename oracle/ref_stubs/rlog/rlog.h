// Minimal stand-in for rlog used only to compile the reference solver as a
// CPU oracle: every log message is discarded.
#ifndef ORACLE_STUB_RLOG_H
#define ORACLE_STUB_RLOG_H
namespace rlog { class RLogChannel; }
#define LOGID 0
#define RLOG_CHANNEL(name) ((rlog::RLogChannel*)0)
#define _rMessage(...) ((void)0)
#endif
