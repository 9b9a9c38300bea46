// Implementation of the HDF5 stand-in (see H5Cpp.h).  Container format,
// little-endian: "AFQH5SH1", uint64 count, then per dataset: uint64 name
// length, name bytes, uint64 rank, rank x uint64 dims, uint64 byte count,
// the bytes (native layout, column-major as the reference stores tensors).
#include "H5Cpp.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>

#include <unistd.h>

namespace H5 {

const PredType PredType::NATIVE_ULONG(8), PredType::NATIVE_DOUBLE(8), PredType::STD_U64BE(8),
    PredType::IEEE_F64BE(8), PredType::NATIVE_INT(4);

static void die(const std::string &m)
{
    std::cerr << "HDF5 stand-in: " << m << std::endl;
    std::exit(1);
}

DataSpace DataSet::getSpace() const
{
    DataSpace s;
    s.dims_ = e_->dims;
    return s;
}

void DataSet::read(void *buf, const DataType &type) const
{
    hsize_t c = 1;
    for (hsize_t d : e_->dims) c *= d;
    if (c * type.getSize() != e_->bytes.size()) die("element size of a read does not match the dataset");
    std::memcpy(buf, e_->bytes.data(), e_->bytes.size());
}

void DataSet::write(const void *buf, const DataType &type)
{
    hsize_t c = 1;
    for (hsize_t d : e_->dims) c *= d;
    e_->bytes.assign((const char *)buf, (const char *)buf + c * type.getSize());
}

H5File::H5File(const std::string &name, unsigned flags)
    : name_(name), data_(std::make_shared<std::map<std::string, Entry>>())
{
    if (flags == H5F_ACC_TRUNC) { dirty_ = true; return; }
    std::ifstream f(name, std::ios::binary);
    if (!f) die("cannot open " + name);
    char magic[8];
    f.read(magic, 8);
    if (std::memcmp(magic, "AFQH5SH1", 8) != 0) die(name + " is not a stand-in container");
    uint64_t n = 0;
    f.read((char *)&n, 8);
    for (uint64_t k = 0; k < n; ++k) {
        uint64_t len = 0, rank = 0, nb = 0;
        f.read((char *)&len, 8);
        std::string key(len, '\0');
        f.read(&key[0], (std::streamsize)len);
        f.read((char *)&rank, 8);
        Entry e;
        e.dims.resize(rank);
        for (uint64_t r = 0; r < rank; ++r) f.read((char *)&e.dims[r], 8);
        f.read((char *)&nb, 8);
        e.bytes.resize(nb);
        f.read(e.bytes.data(), (std::streamsize)nb);
        if (!f) die("truncated container " + name);
        (*data_)[key] = std::move(e);
    }
    if (flags == H5F_ACC_RDWR) { dirty_ = true; opened_ = *data_; }
}

H5File::~H5File() { close(); }

DataSet H5File::openDataSet(const std::string &name) const
{
    auto it = data_->find(name);
    if (it == data_->end()) die("no dataset " + name + " in " + name_);
    return DataSet(&it->second);
}

DataSet H5File::createDataSet(const std::string &name, const DataType &, const DataSpace &space)
{
    Entry &e = (*data_)[name];
    e.dims = space.dims_;
    e.bytes.clear();
    dirty_ = true;
    return DataSet(&e);
}

void H5File::close()
{
    if (!open_) return;
    open_ = false;
    if (!dirty_) return;
    // a read-write open that changed nothing leaves the file as it was
    if (!opened_.empty() && opened_ == *data_) return;
    // written beside the target, then renamed over it: a reader that opened
    // the old container (another program sharing it) never sees a torn file
    const std::string tmp = name_ + ".tmp." + std::to_string((long long)getpid());
    std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
    f.write("AFQH5SH1", 8);
    uint64_t n = data_->size();
    f.write((const char *)&n, 8);
    for (auto &kv : *data_) {
        uint64_t len = kv.first.size(), rank = kv.second.dims.size(), nb = kv.second.bytes.size();
        f.write((const char *)&len, 8);
        f.write(kv.first.data(), (std::streamsize)len);
        f.write((const char *)&rank, 8);
        for (hsize_t d : kv.second.dims) f.write((const char *)&d, 8);
        f.write((const char *)&nb, 8);
        f.write(kv.second.bytes.data(), (std::streamsize)nb);
    }
    f.close();
    if (!f || std::rename(tmp.c_str(), name_.c_str()) != 0) die("cannot write " + name_);
}

}  // namespace H5

int H5Lexists(hid_t file, const char *name, int)
{
    return ((const H5::H5File *)(size_t)file)->exists(name) ? 1 : 0;
}

int H5Ldelete(hid_t file, const char *name, int)
{
    ((H5::H5File *)(size_t)file)->remove(name);
    return 0;
}
