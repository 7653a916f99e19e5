// Minimal stand-in for yaml-cpp, used only to compile the reference sources
// into the CPU oracle (oracle/_ref).  The reference includes "yaml-cpp/yaml.h"
// solely for the inline YAML::convert<> specialisations in its headers
// (Integrator/Statistics.hh, Integrator/Vegas.hh, Channel/MultiChannel.hh);
// none of them is called on the integration path.  This header gives those
// specialisations something to parse.  It is test infrastructure only.
#pragma once

#include <cstddef>
#include <string>
#include <vector>

namespace YAML {

enum class EmitterStyle { Default, Block, Flow };

template <class T> struct convert;

class Node {
  public:
    Node() = default;
    template <class T> Node(const T &) {}
    template <class T> Node &operator=(const T &) { return *this; }
    Node operator[](const std::string &) const { return Node{}; }
    Node operator[](std::size_t) const { return Node{}; }
    Node operator[](int) const { return Node{}; }
    template <class T> T as() const { return T{}; }
    template <class T> void push_back(const T &) {}
    std::size_t size() const { return 0; }
    bool IsSequence() const { return false; }
    void SetStyle(EmitterStyle) {}
    const Node *begin() const { return nullptr; }
    const Node *end() const { return nullptr; }
};

}  // namespace YAML
