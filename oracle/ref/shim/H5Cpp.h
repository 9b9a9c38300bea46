// Stand-in for the subset of the HDF5 C++ API that the reference's
// model/file code uses (common/readWriteHao/source/readWriteHdf5.cpp,
// common/hdf5Hao/source/hdf5CustomHao.cpp, the models' read/write): files
// of named datasets of native 8- and 16-byte elements, kept in a plain
// binary container (written by oracle/ref/ref_run.py for the inputs).  Part
// of the oracle's reference build (test infrastructure only).
#pragma once
#include <cstddef>
#include <map>
#include <memory>
#include <string>
#include <vector>

typedef unsigned long long hsize_t;
typedef long long hid_t;
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_RDWR 1u
#define H5F_ACC_TRUNC 2u
#define H5P_DEFAULT 0
#define HOFFSET(s, m) offsetof(s, m)

namespace H5 {

class DataType {
public:
    explicit DataType(size_t size = 0) : size_(size) {}
    size_t getSize() const { return size_; }

protected:
    size_t size_;
};

class PredType : public DataType {
public:
    explicit PredType(size_t size) : DataType(size) {}
    static const PredType NATIVE_ULONG, NATIVE_DOUBLE, STD_U64BE, IEEE_F64BE, NATIVE_INT;
};

class CompType : public DataType {
public:
    explicit CompType(size_t size) : DataType(size) {}
    void insertMember(const std::string &, size_t, const DataType &) {}
};

class DataSpace {
public:
    DataSpace() = default;
    DataSpace(int rank, const hsize_t *dims) : dims_(dims, dims + rank) {}
    int getSimpleExtentNdims() const { return (int)dims_.size(); }
    int getSimpleExtentDims(hsize_t *dims) const
    {
        for (size_t i = 0; i < dims_.size(); ++i) dims[i] = dims_[i];
        return (int)dims_.size();
    }
    hsize_t count() const
    {
        hsize_t c = 1;
        for (hsize_t d : dims_) c *= d;
        return c;
    }
    std::vector<hsize_t> dims_;
};

struct Entry {
    std::vector<hsize_t> dims;
    std::vector<char> bytes;
    bool operator==(const Entry &o) const { return dims == o.dims && bytes == o.bytes; }
};

class DataSet {
public:
    DataSet() = default;
    explicit DataSet(Entry *e) : e_(e) {}
    DataSpace getSpace() const;
    void read(void *buf, const DataType &type) const;
    void write(const void *buf, const DataType &type);

private:
    Entry *e_ = nullptr;
};

class H5File {
public:
    H5File(const std::string &name, unsigned flags);
    ~H5File();
    DataSet openDataSet(const std::string &name) const;
    DataSet createDataSet(const std::string &name, const DataType &type, const DataSpace &space);
    void close();
    hid_t getId() const { return (hid_t)(size_t)this; }
    bool exists(const std::string &name) const { return data_->count(name) != 0; }
    void remove(const std::string &name) { data_->erase(name); }

private:
    std::string name_;
    bool dirty_ = false, open_ = true;
    std::shared_ptr<std::map<std::string, Entry>> data_;
    std::map<std::string, Entry> opened_;   // contents when opened read-write
};

}  // namespace H5

// H5Lexists / H5Ldelete on an H5File's id
int H5Lexists(hid_t file, const char *name, int plist);
int H5Ldelete(hid_t file, const char *name, int plist);
