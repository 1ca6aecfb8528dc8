// Stand-in for the OCTA/GOURMET `udfmanager.h` (an external library that the
// reference links as `-lplatform`; it is not part of the reference tree and is
// not installed here).  It lets the unmodified reference sources compile so the
// reference itself can serve as the parity oracle.
//
// The stand-in is NOT a UDF parser.  It reads a flat text file of
//     <udf.path> = <value>
// lines keyed by the same UDF paths that the reference asks for through
// `UDFManager::get` (e.g. `mesh.NPX = 5`,
// `object_type.spherical_particle.Particle_spec[0].Particle_number = 2`).
// `put` records values in memory; `write` writes them to the file named at
// construction as the same key lines (the restart file of Save_Restart_udf,
// resume.cxx:10-74, can then be read back as an input), and after
// `newRecord` (Output_udf, output.cxx:268-375) every record's keys are
// written with the prefix `record[<n>].`.
// A `get` of a missing key prints the key to stderr and returns false (the
// reference probes optional keys this way, input.cxx:667-675); the key files
// used here are checked to produce no such line for a required key.
#ifndef KAPSEL_REF_UDFMANAGER_STANDIN_H
#define KAPSEL_REF_UDFMANAGER_STANDIN_H

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

class Location {
  public:
    Location() {}
    Location(const std::string &p) : path_(p) {}
    explicit Location(const char *p) : path_(p) {}
    std::string sub(const std::string &name) const { return path_.empty() ? name : path_ + "." + name; }
    void        down(const std::string &name) { path_ = sub(name); }
    void        up() {
        std::string::size_type pos = path_.rfind('.');
        path_                      = (pos == std::string::npos) ? std::string() : path_.substr(0, pos);
    }
    const std::string &str() const { return path_; }
    operator std::string() const { return path_; }

  private:
    std::string path_;
};

class UDFManager {
  public:
    explicit UDFManager(const std::string &file) { load(file); }
    UDFManager(const std::string &file, const std::string & /*def*/, bool /*flag*/) : out_(file) {}
    UDFManager(const std::string &file, const std::string & /*def*/, int /*flag*/) : out_(file) {}
    ~UDFManager() {}

    template <typename T>
    bool get(const std::string &key, T &value) {
        std::map<std::string, std::string>::const_iterator it = kv_.find(key);
        if (it == kv_.end()) {
            std::fprintf(stderr, "udf stand-in: missing key '%s'\n", key.c_str());
            return false;
        }
        std::istringstream in(it->second);
        in >> value;
        return true;
    }
    bool get(const std::string &key, std::string &value) {
        std::map<std::string, std::string>::const_iterator it = kv_.find(key);
        if (it == kv_.end()) {
            std::fprintf(stderr, "udf stand-in: missing key '%s'\n", key.c_str());
            return false;
        }
        value = it->second;
        return true;
    }
    template <typename T>
    void put(const std::string &key, const T &value) {
        std::ostringstream out;
        out.precision(17);
        out << value;
        kv_[key] = out.str();
    }
    // Number of elements of an array path written as "a.b[]": counts the keys
    // "a.b[0]...", "a.b[1]..." present in the file.
    int size(const std::string &array_path) {
        std::string base = array_path;
        if (base.size() >= 2 && base.compare(base.size() - 2, 2, "[]") == 0) base.erase(base.size() - 2);
        int n = 0;
        for (;;) {
            std::ostringstream p;
            p << base << "[" << n << "]";
            std::string                                        prefix = p.str();
            std::map<std::string, std::string>::const_iterator it     = kv_.lower_bound(prefix);
            if (it == kv_.end() || it->first.compare(0, prefix.size(), prefix) != 0) break;
            ++n;
        }
        return n;
    }
    void write() {
        if (out_.empty()) return;
        FILE *f = std::fopen(out_.c_str(), "w");
        if (!f) {
            std::fprintf(stderr, "udf stand-in: cannot write '%s'\n", out_.c_str());
            return;
        }
        if (records_.empty()) {
            for (std::map<std::string, std::string>::const_iterator it = kv_.begin(); it != kv_.end(); ++it)
                std::fprintf(f, "%s = %s\n", it->first.c_str(), it->second.c_str());
        } else {
            records_.push_back(kv_);
            for (size_t r = 1; r < records_.size(); r++)
                for (std::map<std::string, std::string>::const_iterator it = records_[r].begin();
                     it != records_[r].end(); ++it)
                    std::fprintf(f, "record[%zu].%s = %s\n", r - 1, it->first.c_str(), it->second.c_str());
            records_.pop_back();
        }
        std::fclose(f);
    }
    void newRecord() {
        records_.push_back(kv_);
        kv_.clear();
    }
    std::string getEngineName() { return "kapsel"; }
    std::string getEngineVersion() { return "v3"; }

  private:
    void load(const std::string &file) {
        std::ifstream in(file.c_str());
        if (!in) {
            std::fprintf(stderr, "udf stand-in: cannot open '%s'\n", file.c_str());
            std::abort();
        }
        std::string line;
        while (std::getline(in, line)) {
            std::string::size_type hash = line.find('#');
            if (hash != std::string::npos) line.erase(hash);
            std::string::size_type eq = line.find('=');
            if (eq == std::string::npos) continue;
            kv_[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
        }
    }
    static std::string trim(const std::string &s) {
        std::string::size_type b = s.find_first_not_of(" \t\r\n");
        if (b == std::string::npos) return std::string();
        std::string::size_type e = s.find_last_not_of(" \t\r\n");
        return s.substr(b, e - b + 1);
    }
    std::map<std::string, std::string>              kv_;
    std::string                                     out_;
    std::vector<std::map<std::string, std::string> > records_;
};

#endif
