// OpenQASM front end: QASM text -> qsv_gate records.
//
// Follows QCLAB++'s reader (include/qclab/io/QASMFile.hpp:42-167,
// src/io/QASMFile.cpp:16-53, src/io/util.cpp:6-19) rule for rule:
//   - every line is stripped of all whitespace; blank lines and lines that
//     start with "//" are skipped; a line is split into commands at ';';
//   - commands before the quantum register are ignored unless they start
//     with "qreg"; "qreg<name>[<n>]" fixes the register name and size;
//   - every later command is matched by prefix, in this order:
//     h x y z (name+reg), rx( ry( rz( p( (one angle), cx cy cz swap
//     (name+reg); anything else (measure, barrier, creg, ...) is skipped;
//   - qubits are parsed with std::stoi, angles with std::stof / std::stod
//     in the state's precision, so an expression such as "pi/2" is an error
//     (the reference prints "Failed parsing QASM file!" and keeps the gates
//     read so far; here the call returns QSV_ERROR_INVALID_VALUE and the
//     gates read so far).
// Rotation angles are stored as QRotation(theta) does: cos/sin of theta/2
// computed in the state's real type; Phase as QAngle(theta): cos/sin theta.
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include "internal.hpp"

namespace qsv {
namespace {

std::string left_of(std::string& str, const std::string& delim) {
  const auto pos = str.find_first_of(delim);
  if (pos == 0) return "";
  if (pos == std::string::npos) return str;
  std::string l = str.substr(0, pos);
  str = str.substr(pos + 1);
  return l;
}

qsv_gate blank(int kind) {
  qsv_gate g;
  std::memset(&g, 0, sizeof(g));
  g.kind = kind;
  g.qubit1 = -1;
  g.control_state = 1;
  g.param = -1;
  return g;
}

template <typename R>
R read_angle(const std::string& s);
template <> float read_angle<float>(const std::string& s) { return std::stof(s); }
template <> double read_angle<double>(const std::string& s) { return std::stod(s); }

template <typename R>
void set_angle(qsv_gate& g, R theta, bool half) {
  const R t = half ? theta / 2 : theta;
  g.cos = (double)std::cos(t);
  g.sin = (double)std::sin(t);
}

struct Parser {
  bool has_qreg = false;
  int nq = 0;
  std::string reg;
  std::vector<std::string> commands;

  void feed_line(std::string str) {
    std::string s;
    for (char c : str)
      if (!std::isspace(static_cast<unsigned char>(c))) s.push_back(c);
    if (s.empty()) return;
    if (s.compare(0, 2, "//") == 0) return;
    // split at ';' (the reference's split() never terminates on a leading ';'
    // or a command without ';'; on well-formed lines both agree)
    while (!s.empty()) {
      const auto pos = s.find(';');
      std::string cmd = (pos == std::string::npos) ? s : s.substr(0, pos);
      s = (pos == std::string::npos) ? std::string() : s.substr(pos + 1);
      if (cmd.empty()) continue;
      if (!has_qreg) {
        if (cmd.compare(0, 4, "qreg") == 0) {
          cmd = cmd.substr(4);
          reg = left_of(cmd, "[");
          nq = std::stoi(left_of(cmd, "]"));
          has_qreg = true;
        }
      } else {
        commands.push_back(cmd);
      }
    }
  }
};

template <typename R>
bool parse_command(const std::string& reg, std::string command, std::vector<qsv_gate>* out) {
  const size_t n2 = reg.size();
  auto qubit = [](std::string& str) { return std::stoi(left_of(str, "]")); };
  struct C1 { const char* name; int kind; };
  static const C1 consts1[] = {{"h", QSV_HADAMARD}, {"x", QSV_PAULI_X}, {"y", QSV_PAULI_Y},
                               {"z", QSV_PAULI_Z}};
  static const C1 angles1[] = {{"rx", QSV_ROTATION_X}, {"ry", QSV_ROTATION_Y},
                               {"rz", QSV_ROTATION_Z}, {"p", QSV_PHASE}};
  static const C1 consts2[] = {{"cx", QSV_CX}, {"cy", QSV_CY}, {"cz", QSV_CZ},
                               {"swap", QSV_SWAP}};
  for (const C1& c : consts1) {  // parse1const
    const size_t n1 = std::strlen(c.name);
    if (command.compare(0, n1 + n2, std::string(c.name) + reg) == 0) {
      command.erase(0, n1 + n2 + 1);
      qsv_gate g = blank(c.kind);
      g.qubit0 = qubit(command);
      out->push_back(g);
      return true;
    }
  }
  for (const C1& c : angles1) {  // parse1a
    const size_t n1 = std::strlen(c.name);
    if (command.compare(0, n1 + 1, std::string(c.name) + "(") == 0) {
      command.erase(0, n1 + 1);
      const R theta = read_angle<R>(left_of(command, ")"));
      command.erase(0, n2 + 1);
      qsv_gate g = blank(c.kind);
      g.qubit0 = qubit(command);
      set_angle<R>(g, theta, c.kind != QSV_PHASE);
      out->push_back(g);
      return true;
    }
  }
  for (const C1& c : consts2) {  // parse2const
    const size_t n1 = std::strlen(c.name);
    if (command.compare(0, n1 + n2, std::string(c.name) + reg) == 0) {
      command.erase(0, n1 + n2 + 1);
      qsv_gate g = blank(c.kind);
      g.qubit0 = qubit(command);
      command.erase(0, n2 + 2);
      g.qubit1 = qubit(command);
      out->push_back(g);
      return true;
    }
  }
  return false;
}

}  // namespace
}  // namespace qsv

extern "C" qsv_status qsv_parse_qasm(const char* text, qsv_dtype dtype, qsv_gate* gates,
                                     size_t capacity, size_t* count, int* nbQubits) {
  using namespace qsv;
  if (!text || !count || !nbQubits) return fail(QSV_ERROR_INVALID_VALUE, "null argument");
  if (!dtype_valid(dtype)) return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
  *count = 0;
  *nbQubits = 0;
  Parser p;
  std::vector<qsv_gate> out;
  qsv_status status = QSV_SUCCESS;
  try {
    const char* s = text;
    while (*s) {
      const char* e = std::strchr(s, '\n');
      const size_t len = e ? (size_t)(e - s) : std::strlen(s);
      p.feed_line(std::string(s, len));
      s += len + (e ? 1 : 0);
    }
  } catch (const std::exception& ex) {
    return fail(QSV_ERROR_INVALID_VALUE, "QASM register line could not be parsed: %s", ex.what());
  }
  if (!p.has_qreg) return fail(QSV_ERROR_INVALID_VALUE, "QASM text has no qreg");
  *nbQubits = p.nq;
  const bool single = (dtype == QSV_C64 || dtype == QSV_F32);
  try {
    for (const std::string& cmd : p.commands) {
      if (single) parse_command<float>(p.reg, cmd, &out);
      else parse_command<double>(p.reg, cmd, &out);
    }
  } catch (const std::exception& ex) {
    // the reference stops here and keeps the gates read so far
    status = fail(QSV_ERROR_INVALID_VALUE, "failed parsing QASM after %zu gates: %s",
                  out.size(), ex.what());
  }
  for (const qsv_gate& g : out) {
    const int hi = std::max(g.qubit0, g.qubit1);
    if (g.qubit0 < 0 || hi >= p.nq)
      return fail(QSV_ERROR_QUBIT, "QASM gate on qubit %d outside the %d-qubit register", hi, p.nq);
  }
  *count = out.size();
  if (gates && capacity >= out.size())
    std::memcpy(gates, out.data(), out.size() * sizeof(qsv_gate));
  else if (capacity < out.size() && status == QSV_SUCCESS && gates)
    return fail(QSV_ERROR_SIZE, "%zu gates do not fit the %zu-record buffer", out.size(), capacity);
  return status;
}
