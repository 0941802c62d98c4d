// PropertyTree.h -- the subset of an XML property tree the reference's
// configuration and event-list files use (Boost.PropertyTree's XML form:
// nested elements with text, no attributes; IAC/Settings.h:44-86,
// IAC/MainRunModes.cpp:32-91, IAC/Settings.cpp:473-676).  Paths are
// dot-separated element names, e.g. "root.EvalSettings.OutputMesh.MeshSize".
#pragma once

#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace iac {

class PropertyTree {
public:
    std::string name, text;
    std::vector<PropertyTree> children;

    static PropertyTree ReadXml(const std::string &filename);  // throws on I/O or syntax errors
    static PropertyTree ParseXml(const std::string &xml);
    void WriteXml(const std::string &filename) const;
    std::string ToXml() const;

    const PropertyTree *Find(const std::string &path) const;
    PropertyTree &Put(const std::string &path, const std::string &value);  // creates elements

    std::string Get(const std::string &path, const std::string &fallback) const;
    template <typename T>
    T Get(const std::string &path, T fallback) const
    {
        const PropertyTree *n = Find(path);
        if (!n) return fallback;
        std::istringstream is(n->text);
        T v;
        if (!(is >> v)) return fallback;
        return v;
    }
    bool GetBool(const std::string &path, bool fallback) const;
    template <typename T>
    PropertyTree &Put(const std::string &path, T value)
    {
        std::ostringstream os;
        os << value;
        return Put(path, os.str());
    }
};

}  // namespace iac
