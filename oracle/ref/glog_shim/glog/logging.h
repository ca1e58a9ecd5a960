// Test infrastructure only: a project-written stand-in for the one glog
// facility the reference uses (LOG(ERROR) << ..., at
// src/Smoothers/SymmetricGaussSeidelSmoother.cc:63). Writes to stderr.
#pragma once
#include <iostream>
#include <sstream>

namespace glog_shim {
class LogLine {
 public:
  explicit LogLine(const char *severity) { stream_ << "[" << severity << "] "; }
  ~LogLine() { std::cerr << stream_.str() << std::endl; }
  template <typename T>
  LogLine &operator<<(const T &v) { stream_ << v; return *this; }

 private:
  std::ostringstream stream_;
};
}  // namespace glog_shim

#define LOG(severity) ::glog_shim::LogLine(#severity)
