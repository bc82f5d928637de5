// Host-only key/value reader with the calling convention of AMReX's
// ParmParse (query / queryarr under a prefix), used by a case's
// amrex_probinit to read its `prob.*` parameters.  Input is the text of a
// reference inputs file: `prefix.key = v1 v2 ...` lines, `#` comments.
#pragma once

#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace vd {

class ParmParse
{
public:
    using Table = std::map<std::string, std::vector<std::string>>;

    ParmParse(const Table* table, std::string prefix)
        : m_table(table), m_prefix(std::move(prefix))
    {
    }

    static Table parse(const std::string& text)
    {
        Table t;
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line))
        {
            const auto hash = line.find('#');
            if (hash != std::string::npos) line = line.substr(0, hash);
            const auto eq = line.find('=');
            if (eq == std::string::npos) continue;
            std::string key = trim(line.substr(0, eq));
            std::istringstream vs(line.substr(eq + 1));
            std::vector<std::string> vals;
            std::string v;
            while (vs >> v) vals.push_back(v);
            if (!key.empty()) t[key] = vals;
        }
        return t;
    }

    const std::vector<std::string>* find(const std::string& name) const
    {
        if (!m_table) return nullptr;
        auto it = m_table->find(m_prefix.empty() ? name : m_prefix + "." + name);
        return it == m_table->end() ? nullptr : &it->second;
    }

    template <class T>
    bool query(const std::string& name, T& out) const
    {
        auto* v = find(name);
        if (!v || v->empty()) return false;
        std::istringstream s((*v)[0]);
        s >> out;
        return true;
    }

    template <class T>
    bool queryarr(const std::string& name, T* out, int n) const
    {
        auto* v = find(name);
        if (!v) return false;
        for (int i = 0; i < n && i < (int)v->size(); ++i)
        {
            std::istringstream s((*v)[i]);
            s >> out[i];
        }
        return true;
    }

private:
    static std::string trim(const std::string& s)
    {
        const auto b = s.find_first_not_of(" \t\r\n");
        const auto e = s.find_last_not_of(" \t\r\n");
        return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
    }

    const Table* m_table;
    std::string m_prefix;
};

} // namespace vd
