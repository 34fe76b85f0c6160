/*
 * Levelled logger of the class-level API (the reference's logger.h:27-150, logger.cpp:61-62): the same levels,
 * methods and the two process-wide loggers stdLogger and rootLogger (rank 0 only; every process is rank 0 here).
 * Messages are "# <date time> LEVEL: <message>".
 */
#ifndef LOGGER_H
#define LOGGER_H

#include <ctime>
#include <iostream>
#include <sstream>
#include <string>

#include "kuqcd_utils.h"

namespace kuqcd {

enum class LogLevel { ALL, ALLOC, TRACE, DEBUG, INFO, WARN, ERROR, FATAL, OFF };

class Logger {
public:
    explicit Logger(LogLevel level = LogLevel::ALL, bool colorized = true, std::ostream &out = std::cout,
                    std::string prefix = "")
        : level_(level), color_(colorized), out_(out), prefix_(std::move(prefix))
    {
    }
    void SetVerbosity(LogLevel v) { level_ = v; }
    LogLevel GetVerbosity() { return level_; }
    void SetColoredOutput(bool v) { color_ = v; }
    void SetAdditionalPrefix(std::string p) { prefix_ = std::move(p); }
    std::string GetAdditionalPrefix() { return prefix_; }

    template <LogLevel L, typename... Args>
    std::string Message(Args &&...args)
    {
        static const char *names[] = {"ALL", "ALLOC", "TRACE", "DEBUG", "INFO", "WARN", "ERROR", "FATAL", "OFF"};
        std::ostringstream msg;
        (msg << ... << args);
        const char *on = !color_ ? "" : L == LogLevel::WARN ? "\033[0;33m" : L >= LogLevel::ERROR ? "\033[0;31m" : "";
        const char *off = *on ? "\033[0m" : "";
        char stamp[32];
        const std::time_t now = std::time(nullptr);
        std::strftime(stamp, sizeof(stamp), "%Y-%m-%d %H:%M:%S ", std::localtime(&now));
        if (L >= level_ && GetRank() == 0)
            out_ << on << "# " << stamp << names[static_cast<int>(L)] << ": " << prefix_ << msg.str() << off
                 << std::endl;
        return prefix_ + msg.str();
    }
    template <typename... Args> std::string Alloc(Args &&...a) { return Message<LogLevel::ALLOC>(a...); }
    template <typename... Args> std::string Trace(Args &&...a) { return Message<LogLevel::TRACE>(a...); }
    template <typename... Args> std::string Debug(Args &&...a) { return Message<LogLevel::DEBUG>(a...); }
    template <typename... Args> std::string Info(Args &&...a) { return Message<LogLevel::INFO>(a...); }
    template <typename... Args> std::string Warn(Args &&...a) { return Message<LogLevel::WARN>(a...); }
    template <typename... Args> std::string Error(Args &&...a) { return Message<LogLevel::ERROR>(a...); }
    template <typename... Args> std::string Fatal(Args &&...a) { return Message<LogLevel::FATAL>(a...); }

private:
    LogLevel level_;
    bool color_;
    std::ostream &out_;
    std::string prefix_;
};

inline Logger stdLogger(LogLevel::INFO);
inline Logger rootLogger(LogLevel::INFO, true, std::cout, "[ROOT] ");

}  // namespace kuqcd

#endif
