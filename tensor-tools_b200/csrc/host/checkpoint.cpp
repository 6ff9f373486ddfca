// MPS checkpoint writer / reader (metadata text file + raw block file).
#include "checkpoint.h"

#include <cstdio>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>

namespace ttb {

namespace {

const char* kQMagic = "tt_b200-qmps-checkpoint 1";
const char* kDMagic = "tt_b200-mps-checkpoint 1";

void check_name(const std::string& s) {
  if (s.empty() || s.find_first_of(" \t\r\n") != std::string::npos)
    throw std::runtime_error("checkpoint: names must be non-empty and contain no whitespace: '" + s + "'");
}

std::string raw_name(const std::string& fn, const std::string& wfn) { return wfn.empty() ? fn + "__T.bin" : wfn; }

struct RawFile {
  std::FILE* f = nullptr;
  RawFile(const std::string& path, const char* mode) : f(std::fopen(path.c_str(), mode)) {
    if (!f) throw std::runtime_error("checkpoint: cannot open " + path);
  }
  ~RawFile() {
    if (f) std::fclose(f);
  }
  void close(const std::string& path) {
    const bool bad = std::ferror(f) != 0;
    const int rc = std::fclose(f);
    f = nullptr;
    if (bad || rc != 0) throw std::runtime_error("checkpoint: cannot write " + path);
  }
  void write(const double* p, size_t n) {
    if (n && std::fwrite(p, sizeof(double), n, f) != n) throw std::runtime_error("checkpoint: short write");
  }
  void read(int64_t byte_off, double* p, size_t n) {
    if (std::fseek(f, (long)byte_off, SEEK_SET) != 0) throw std::runtime_error("checkpoint: seek failed");
    if (n && std::fread(p, sizeof(double), n, f) != n) throw std::runtime_error("checkpoint: raw file too short");
  }
};

std::vector<double> download(const double* dev, int64_t n) {
  std::vector<double> h((size_t)n);
  if (n) check(tt_memcpy_d2h(rt().ctx, h.data(), dev, sizeof(double) * (size_t)n), "checkpoint download");
  return h;
}

void upload(double* dev, const std::vector<double>& h) {
  if (!h.empty()) check(tt_memcpy_h2d(rt().ctx, dev, h.data(), sizeof(double) * h.size()), "checkpoint upload");
  check(tt_ctx_synchronize(rt().ctx), "checkpoint sync");
}

// A save writes both files under temporary names and renames each into place,
// the raw block file first and the metadata last: a crash or a full disk
// during a save leaves the previous checkpoint whole.
void commit_file(const std::string& tmp, const std::string& path) {
  if (std::rename(tmp.c_str(), path.c_str()) != 0) throw std::runtime_error("checkpoint: cannot rename " + tmp);
}

void write_meta(const std::string& fn, const std::string& meta) {
  const std::string path = fn + ".ttmps", tmp = path + ".tmp";
  {
    std::ofstream out(tmp);
    out << meta;
    out.flush();
    if (!out) throw std::runtime_error("checkpoint: cannot write " + tmp);
  }
  commit_file(tmp, path);
}

// the raw file named in the metadata: a relative name is taken under
// data_prefix, an absolute one as it stands
std::string raw_path(const std::string& data_prefix, const std::string& wfn) {
  return !wfn.empty() && wfn[0] == '/' ? wfn : data_prefix + wfn;
}

std::string expect(std::istream& in, const char* key) {
  std::string k;
  if (!(in >> k) || k != key) throw std::runtime_error(std::string("checkpoint: expected '") + key + "'");
  return k;
}

}  // namespace

// ---- qMPS ---------------------------------------------------------------------
void save(const qMPS& psi, const std::string& fn, const std::string& wfn_in) {
  if (!rt().ctx) throw std::runtime_error("checkpoint: no device context bound");
  const std::string wfn = raw_name(fn, wfn_in);
  std::ostringstream meta;
  meta.precision(17);
  meta << kQMagic << "\n";
  meta << "wfn " << wfn << "\n";
  meta << "length " << psi.length << "\nphy_dim " << psi.phy_qn.size() << "\nid " << psi.id << "\ncenter "
       << psi.center << "\n";
  meta << "totalQ " << psi.totalQ.a << " " << psi.totalQ.b << "\n";
  meta << "phy_qn " << psi.phy_qn.size();
  for (auto& q : psi.phy_qn) meta << " " << q.a << " " << q.b;
  meta << "\nbond_dims " << psi.bond_dims.size();
  for (auto d : psi.bond_dims) meta << " " << d;
  meta << "\n";
  RawFile raw(wfn + ".tmp", "wb");
  int64_t offset = 0;
  for (unsigned i = 0; i < psi.length; ++i) {
    const qtensor& T = psi.A[i];
    meta << "tensor " << i << " rank " << T.rank << " blocks " << T.blocks.size() << "\n";
    for (auto& ix : T.idx_set) {
      check_name(ix.name());
      meta << "index " << (int)ix.arrow() << " " << (int)ix.type() << " " << ix.level() << " " << ix.name() << " "
           << ix.size();
      for (auto& s : ix.sectors()) meta << " " << s.first.a << " " << s.first.b << " " << s.second;
      meta << "\n";
    }
    std::vector<double> h = download(T.arena ? T.data->get() : nullptr, T.arena);
    for (auto& b : T.blocks) {
      meta << "block";
      for (unsigned q : b.qi) meta << " " << q;
      meta << " " << offset << "\n";
      raw.write(h.data() + b.off, (size_t)b.size);
      offset += b.size * (int64_t)sizeof(double);
    }
  }
  raw.close(wfn + ".tmp");
  commit_file(wfn + ".tmp", wfn);
  write_meta(fn, meta.str());
}

qMPS load_qmps(const std::string& fn, const std::string& data_prefix) {
  if (!rt().ctx) throw std::runtime_error("checkpoint: no device context bound");
  std::ifstream in(fn);
  if (!in) throw std::runtime_error("checkpoint: cannot open " + fn);
  std::string line;
  std::getline(in, line);
  if (line != kQMagic) throw std::runtime_error("checkpoint: not a qMPS checkpoint: " + fn);
  qMPS psi;
  std::string wfn;
  unsigned phy_dim = 0;
  size_t n = 0;
  expect(in, "wfn");
  in >> wfn;
  expect(in, "length");
  in >> psi.length;
  expect(in, "phy_dim");
  in >> phy_dim;
  expect(in, "id");
  in >> psi.id;
  expect(in, "center");
  in >> psi.center;
  expect(in, "totalQ");
  in >> psi.totalQ.a >> psi.totalQ.b;
  expect(in, "phy_qn");
  in >> n;
  psi.phy_qn.resize(n);
  for (auto& q : psi.phy_qn) in >> q.a >> q.b;
  expect(in, "bond_dims");
  in >> n;
  psi.bond_dims.resize(n);
  for (auto& d : psi.bond_dims) in >> d;
  if (!in || psi.length < 2 || psi.bond_dims.size() != psi.length + 1 || phy_dim != psi.phy_qn.size())
    throw std::runtime_error("checkpoint: bad qMPS header in " + fn);
  RawFile raw(raw_path(data_prefix, wfn), "rb");
  for (unsigned i = 0; i < psi.length; ++i) {
    unsigned ti = 0, rank = 0;
    size_t nb = 0;
    expect(in, "tensor");
    in >> ti;
    expect(in, "rank");
    in >> rank;
    expect(in, "blocks");
    in >> nb;
    if (!in || ti != i || rank == 0 || rank > 8) throw std::runtime_error("checkpoint: bad tensor record");
    std::vector<qtensor_index> idx;
    for (unsigned k = 0; k < rank; ++k) {
      int arrow = 0, type = 0;
      unsigned level = 0, nsec = 0;
      std::string name;
      expect(in, "index");
      in >> arrow >> type >> level >> name >> nsec;
      qtensor_index ix(arrow == 0 ? Inward : Outward, name, type == 0 ? Link : Site, level);
      for (unsigned s = 0; s < nsec; ++s) {
        int32_t a = 0, b = 0;
        unsigned d = 0;
        in >> a >> b >> d;
        ix.addQN(QN(a, b), d);
      }
      if (!in || ix.size() != nsec) throw std::runtime_error("checkpoint: bad index record");
      idx.push_back(ix);
    }
    qtensor T(idx);
    std::vector<int64_t> offs;
    for (size_t b = 0; b < nb; ++b) {
      expect(in, "block");
      std::vector<unsigned> qi(rank);
      std::vector<QN> qn(rank);
      std::vector<int> qd(rank);
      for (unsigned k = 0; k < rank; ++k) {
        in >> qi[k];
        if (!in || qi[k] >= T.idx_set[k].size()) throw std::runtime_error("checkpoint: bad block record");
        qn[k] = T.idx_set[k].qn(qi[k]);
        qd[k] = (int)T.idx_set[k].qdim(qi[k]);
      }
      int64_t off = 0;
      in >> off;
      if (!in || off < 0) throw std::runtime_error("checkpoint: bad block offset");
      T.add_block_meta(qn, qi, qd);
      offs.push_back(off);
    }
    T.allocate(false);
    T._initted = true;
    std::vector<double> h((size_t)T.arena);
    for (size_t b = 0; b < nb; ++b) raw.read(offs[b], h.data() + T.blocks[b].off, (size_t)T.blocks[b].size);
    if (T.arena) upload(T.data->get(), h);
    psi.A.push_back(std::move(T));
  }
  return psi;
}

// ---- dense MPS -------------------------------------------------------------------
void save(const MPS& psi, const std::string& fn, const std::string& wfn_in) {
  if (!rt().ctx) throw std::runtime_error("checkpoint: no device context bound");
  const std::string wfn = raw_name(fn, wfn_in);
  std::ostringstream meta;
  meta << kDMagic << "\n";
  meta << "wfn " << wfn << "\n";
  meta << "length " << psi.length << "\nphy_dim " << psi.phy_dim << "\nid " << psi.id << "\ncenter " << psi.center
       << "\n";
  meta << "bond_dims " << psi.bond_dims.size();
  for (auto d : psi.bond_dims) meta << " " << d;
  meta << "\n";
  RawFile raw(wfn + ".tmp", "wb");
  int64_t offset = 0;
  for (unsigned i = 0; i < psi.length; ++i) {
    const dtensor& T = psi.A[i];
    meta << "tensor " << i << " rank " << T.rank << " offset " << offset << "\n";
    for (auto& ix : T.idx_set) {
      check_name(ix.name);
      meta << "index " << (int)ix.type << " " << ix.level << " " << ix.name << " " << ix.size << "\n";
    }
    std::vector<double> h = download(T.data->get(), T.size);
    raw.write(h.data(), h.size());
    offset += T.size * (int64_t)sizeof(double);
  }
  raw.close(wfn + ".tmp");
  commit_file(wfn + ".tmp", wfn);
  write_meta(fn, meta.str());
}

MPS load_mps(const std::string& fn, const std::string& data_prefix) {
  if (!rt().ctx) throw std::runtime_error("checkpoint: no device context bound");
  std::ifstream in(fn);
  if (!in) throw std::runtime_error("checkpoint: cannot open " + fn);
  std::string line;
  std::getline(in, line);
  if (line != kDMagic) throw std::runtime_error("checkpoint: not a dense MPS checkpoint: " + fn);
  MPS psi;
  std::string wfn;
  size_t n = 0;
  expect(in, "wfn");
  in >> wfn;
  expect(in, "length");
  in >> psi.length;
  expect(in, "phy_dim");
  in >> psi.phy_dim;
  expect(in, "id");
  in >> psi.id;
  expect(in, "center");
  in >> psi.center;
  expect(in, "bond_dims");
  in >> n;
  psi.bond_dims.resize(n);
  for (auto& d : psi.bond_dims) in >> d;
  if (!in || psi.length < 2 || psi.bond_dims.size() != psi.length + 1)
    throw std::runtime_error("checkpoint: bad MPS header in " + fn);
  RawFile raw(raw_path(data_prefix, wfn), "rb");
  for (unsigned i = 0; i < psi.length; ++i) {
    unsigned ti = 0, rank = 0;
    int64_t off = 0;
    expect(in, "tensor");
    in >> ti;
    expect(in, "rank");
    in >> rank;
    expect(in, "offset");
    in >> off;
    if (!in || ti != i || rank == 0 || rank > 8 || off < 0) throw std::runtime_error("checkpoint: bad tensor record");
    std::vector<dtensor_index> idx;
    for (unsigned k = 0; k < rank; ++k) {
      int type = 0;
      unsigned level = 0;
      int64_t size = 0;
      std::string name;
      expect(in, "index");
      in >> type >> level >> name >> size;
      if (!in || size <= 0) throw std::runtime_error("checkpoint: bad index record");
      idx.emplace_back(size, name, type == 0 ? Link : Site, level);
    }
    dtensor T(idx, false);
    std::vector<double> h((size_t)T.size);
    raw.read(off, h.data(), h.size());
    upload(T.data->get(), h);
    psi.A.push_back(std::move(T));
  }
  return psi;
}

}  // namespace ttb
