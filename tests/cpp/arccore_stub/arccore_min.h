// arccore_min.h -- TEST INFRASTRUCTURE.  The few Arccore declarations that
// Alien's own headers on the back-end boundary need in order to compile
// without Arccore (absent here; Alien's build fetches it at configure time):
// the ones named by alien/utils/Precomp.h and alien/utils/arccore/AlienTypes.h
// (type aliases, String, array views, exceptions with A_FUNCINFO, the trace
// manager) and by expression/solver/SolverStat.cc (trace listeners).  Class
// templates the Alien headers use only inside their own templates are
// declared, not defined.  Every header under arccore/ in this directory
// forwards here.  A real build uses Arccore itself.
#pragma once

#include <cstdint>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>

namespace Arccore {

using Byte = unsigned char;
using Int32 = std::int32_t;
using Int64 = std::int64_t;
using Integer = Int32;
using Real = double;

class String {
 public:
  String() = default;
  String(const char* s) : m_s(s ? s : ""), m_null(s == nullptr) {}
  String(const std::string& s) : m_s(s), m_null(false) {}
  const char* localstr() const { return m_s.c_str(); }
  bool null() const { return m_null; }
  bool empty() const { return m_s.empty(); }
  bool operator==(const String& o) const { return m_s == o.m_s; }
  template <typename... U>
  static String format(const String& f, const U&...) {
    return f;
  }
  friend std::ostream& operator<<(std::ostream& o, const String& s) { return o << s.m_s; }

 private:
  std::string m_s;
  bool m_null = true;
};

template <typename T>
class ConstArrayView {
 public:
  ConstArrayView() = default;
  ConstArrayView(Integer n, const T* p) : m_p(p), m_n(n) {}
  Integer size() const { return m_n; }
  const T& operator[](Integer i) const { return m_p[i]; }
  const T* data() const { return m_p; }
  const T* begin() const { return m_p; }
  const T* end() const { return m_p + m_n; }

 private:
  const T* m_p = nullptr;
  Integer m_n = 0;
};

template <typename T>
class ArrayView {
 public:
  ArrayView() = default;
  ArrayView(Integer n, T* p) : m_p(p), m_n(n) {}
  Integer size() const { return m_n; }
  T& operator[](Integer i) const { return m_p[i]; }
  T* data() const { return m_p; }
  T* begin() const { return m_p; }
  T* end() const { return m_p + m_n; }

 private:
  T* m_p = nullptr;
  Integer m_n = 0;
};

template <typename T>
class UniqueArray;
template <typename T>
class SharedArray;
template <typename T>
class UniqueArray2;
template <typename T>
class SharedArray2;
template <typename T>
class Array2View;
template <typename T>
class ConstArray2View;
template <typename T>
class Ref;
class ISerializer;
class TraceMessage;

namespace MessagePassing {
class IMessagePassingMng;
class MessageRank;
class ISerializeMessage;
class ISerializeMessageList;
}  // namespace MessagePassing

class TraceInfo {
 public:
  TraceInfo(const char* file, const char* func, int line) : m_file(file), m_func(func), m_line(line) {}
  const char* file() const { return m_file; }
  const char* name() const { return m_func; }
  int line() const { return m_line; }

 private:
  const char* m_file;
  const char* m_func;
  int m_line;
};

class Exception : public std::runtime_error {
 public:
  Exception(const char* kind, const TraceInfo& where, const String& message)
      : std::runtime_error(std::string(kind) + " in " + where.name() + ": " + message.localstr()) {}
};

class ArgumentException : public Exception {
 public:
  ArgumentException(const TraceInfo& where, const String& message) : Exception("ArgumentException", where, message) {}
};
class FatalErrorException : public Exception {
 public:
  FatalErrorException(const TraceInfo& where, const String& message)
      : Exception("FatalErrorException", where, message) {}
};
class NotImplementedException : public Exception {
 public:
  NotImplementedException(const TraceInfo& where, const String& message)
      : Exception("NotImplementedException", where, message) {}
};

class TraceMessageListenerArgs {
 public:
  explicit TraceMessageListenerArgs(ConstArrayView<char> buf) : m_buf(buf) {}
  ConstArrayView<char> buffer() const { return m_buf; }

 private:
  ConstArrayView<char> m_buf;
};

class ITraceMessageListener {
 public:
  virtual ~ITraceMessageListener() = default;
  virtual bool visitMessage(const TraceMessageListenerArgs& args) = 0;
};

// info() hands out a stream; listeners see nothing (no message prefix).
class ITraceMng {
 public:
  virtual ~ITraceMng() = default;
  virtual std::ostream& info() = 0;
  virtual void addListener(ITraceMessageListener*) {}
  virtual void removeListener(ITraceMessageListener*) {}
};

}  // namespace Arccore

#define A_FUNCINFO ::Arccore::TraceInfo(__FILE__, __func__, __LINE__)
