// json/writer.h -- the part of jsoncpp's Json::Value the reference's solver
// headers name (fillInfo signatures, src/solver2D.cpp:121-124).  TEST
// INFRASTRUCTURE ONLY (reference pin build): values are accepted and
// discarded; the pin never writes JSON.
#ifndef PXP_REFSHIM_JSON_WRITER_H
#define PXP_REFSHIM_JSON_WRITER_H
#include <string>

namespace Json {
class Value {
 public:
  Value() = default;
  template <typename T> Value(const T &) {}
  template <typename T> Value &operator=(const T &) { return *this; }
  Value &operator[](const char *) { return *this; }
  Value &operator[](const std::string &) { return *this; }
  Value &operator[](int) { return *this; }
  Value &append(const Value &) { return *this; }
};
}  // namespace Json
#endif
