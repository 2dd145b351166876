// H5Cpp.h -- the declarations of the HDF5 C++ API that the reference's
// ParaxialSimulation names (src/paraxialSimulation.cpp:137-193, 285-353,
// 454-511).  TEST INFRASTRUCTURE ONLY (reference pin build): the pin steps
// solvers and reads their arrays; it never saves.  Opening a file throws, so
// an HDF5 write cannot pass silently.
#ifndef PXP_REFSHIM_H5CPP_H
#define PXP_REFSHIM_H5CPP_H
#include <stdexcept>
#include <string>

typedef long long hid_t;
typedef unsigned long long hsize_t;
#define H5F_ACC_TRUNC 2u
enum H5S_class_t { H5S_SCALAR = 0, H5S_SIMPLE = 1 };

namespace H5 {
typedef std::string H5std_string;

class PredType {
 public:
  explicit PredType(int id = 0) : id_(id) {}
  bool operator==(const PredType &o) const { return id_ == o.id_; }
  bool operator!=(const PredType &o) const { return id_ != o.id_; }
  static const PredType NATIVE_DOUBLE, NATIVE_INT, NATIVE_UINT8, C_S1;

 private:
  int id_;
};
inline const PredType PredType::NATIVE_DOUBLE{1};
inline const PredType PredType::NATIVE_INT{2};
inline const PredType PredType::NATIVE_UINT8{3};
inline const PredType PredType::C_S1{4};

class StrType {
 public:
  StrType(const PredType &, size_t) {}
};

class DataSpace {
 public:
  explicit DataSpace(H5S_class_t) {}
  DataSpace(int, const hsize_t *) {}
};

class Attribute {
 public:
  void write(const PredType &, const void *) const {}
  void write(const StrType &, const H5std_string &) const {}
};

class DataSet {
 public:
  Attribute createAttribute(const char *, const PredType &, const DataSpace &) const { return {}; }
  void write(const void *, const PredType &) const {}
};

class Group {
 public:
  Attribute createAttribute(const char *, const PredType &, const DataSpace &) const { return {}; }
  Attribute createAttribute(const char *, const StrType &, const DataSpace &) const { return {}; }
};

class H5File {
 public:
  H5File(const char *, unsigned) {
    throw std::runtime_error("HDF5 is not available in the reference pin build");
  }
  H5File(const std::string &n, unsigned f) : H5File(n.c_str(), f) {}
  Group createGroup(const std::string &) const { return {}; }
  DataSet createDataSet(const std::string &, const PredType &, const DataSpace &) const {
    return {};
  }
};
}  // namespace H5
using H5::H5std_string;
#endif
