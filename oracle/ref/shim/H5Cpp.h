// Build shim: no-op stand-ins for the few HDF5 C++ names that
// IMRTBeamBundle.cu mentions in doseDataSave (never called by the harness).
#pragma once
#include <string>
typedef unsigned long long hsize_t;
#define H5F_ACC_TRUNC 0
namespace H5 {
struct PredType { static const int NATIVE_INT = 0; static const int NATIVE_FLOAT = 1; };
struct DataSpace { DataSpace(int, const hsize_t*) {} };
struct DataSet { void write(const void*, int) {} void close() {} };
struct H5File {
    H5File(const std::string&, int) {}
    DataSet createDataSet(const char*, int, const DataSpace&) { return DataSet(); }
};
}
