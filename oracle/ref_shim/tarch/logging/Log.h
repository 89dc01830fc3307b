#pragma once
#include <iostream>
#include <string>
namespace tarch { namespace logging {
class Log { public: explicit Log(const std::string&) {} };
}}
#define logWarning(method, msg) do { std::cerr << "warning " << method << ": " << msg << std::endl; } while (0)
#define logInfo(method, msg) do {} while (0)
#define logDebug(method, msg) do {} while (0)
#define logError(method, msg) do { std::cerr << "error " << method << ": " << msg << std::endl; } while (0)
