// tg_mesh.cc -- host construction of the device mesh layout (see tg_mesh.h).
#include "tg_mesh.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <unordered_map>

namespace tg {

namespace {

// Position along a Hilbert curve on a 2^16 x 2^16 grid.
uint64_t hilbert_index(uint32_t x, uint32_t y) {
  const uint32_t n = 1u << 16;
  uint64_t d = 0;
  for (uint32_t s = n / 2; s > 0; s /= 2) {
    uint32_t rx = (x & s) ? 1u : 0u;
    uint32_t ry = (y & s) ? 1u : 0u;
    d += (uint64_t)s * (uint64_t)s * (uint64_t)((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = n - 1 - x;
        y = n - 1 - y;
      }
      std::swap(x, y);
    }
  }
  return d;
}

struct Err {
  std::string msg;
  bool bad() const { return !msg.empty(); }
};

}  // namespace

std::string build_layout(const tg_mesh& m, const tg_bc_table* bc, bool need_viscous, HostLayout& L) {
  char buf[256];
  const int nv = m.n_vertex, nc = m.n_cell, nf = m.n_face, nbf = m.n_bface;
  if (nv <= 0 || nc <= 0 || nf <= 0 || nbf < 0) return "mesh has no vertices, cells or faces";
  if (!m.coords || !m.dcarea || !m.mcarea || !m.cell_vertex || !m.cell_normal || !m.cell_area ||
      !m.face_vertex || !m.face_type || !m.face_normal || !m.face_lcell || !m.face_rcell)
    return "mesh array pointer is NULL";
  if (nbf > 0 && (!m.bface_vertex || !m.bface_type || !m.bface_normal || !m.bface_lcell || !m.bface_periodic))
    return "boundary-face array pointer is NULL";
  if (nbf > nf) return "more boundary faces than faces";
  for (int i = 0; i < 2 * nf; ++i)
    if (m.face_vertex[i] < 0 || m.face_vertex[i] >= nv) return "face vertex index out of range";
  for (int i = 0; i < nf; ++i) {
    if (m.face_lcell[i] < 0 || m.face_lcell[i] >= nc) return "face left cell out of range";
    if (m.face_rcell[i] >= nc) return "face right cell out of range";
    if (m.face_type[i] == -2) return "inter-partition faces (type -2) need more than one partition";
  }
  for (int i = 0; i < 3 * nc; ++i)
    if (m.cell_vertex[i] < 0 || m.cell_vertex[i] >= nv) return "cell vertex index out of range";
  for (int b = 0; b < nbf; ++b) {
    if (m.bface_vertex[2 * b] < 0 || m.bface_vertex[2 * b] >= nv || m.bface_vertex[2 * b + 1] < 0 ||
        m.bface_vertex[2 * b + 1] >= nv)
      return "boundary-face vertex index out of range";
    if (m.bface_lcell[b] < 0 || m.bface_lcell[b] >= nc) return "boundary-face cell out of range";
    // Boundary faces lead the face list: face[b] is bface[b] (src/grid_preproc.cc:530-541).
    int a0 = m.face_vertex[2 * b], a1 = m.face_vertex[2 * b + 1];
    int b0 = m.bface_vertex[2 * b], b1 = m.bface_vertex[2 * b + 1];
    if (m.face_type[b] != m.bface_type[b] || !((a0 == b0 && a1 == b1) || (a0 == b1 && a1 == b0))) {
      std::snprintf(buf, sizeof(buf), "face %d does not match boundary face %d (boundary faces must lead the face list)", b, b);
      return buf;
    }
  }
  for (int i = 0; i < nv; ++i)
    if (!(m.dcarea[i] > 0.0) || !(m.mcarea[i] > 0.0)) return "non-positive dual area";
  const bool axi = m.vertex_radius || m.face_radius || m.cell_radius;
  if (axi && !(m.vertex_radius && m.face_radius && m.cell_radius))
    return "an axisymmetric mesh needs vertex, face and cell radii";

  // periodic sets -> set id per vertex
  std::vector<int> set_of(nv, -1);
  const int np = m.n_periodic;
  if (np > 0 && (!m.periodic_offsets || !m.periodic_members)) return "periodic list pointer is NULL";
  for (int s = 0; s < np; ++s) {
    if (m.periodic_offsets[s + 1] <= m.periodic_offsets[s]) return "empty periodic set";
    for (int j = m.periodic_offsets[s]; j < m.periodic_offsets[s + 1]; ++j) {
      int v = m.periodic_members[j];
      if (v < 0 || v >= nv) return "periodic vertex out of range";
      if (set_of[v] != -1) return "vertex belongs to two periodic sets";
      set_of[v] = s;
    }
  }

  // boundary-condition lookup
  auto bc_of = [&](int tag, int& kind, int& adiab) {
    kind = 0;
    adiab = 0;
    if (!bc) return false;
    for (int i = 0; i < bc->n_types; ++i)
      if (bc->type_tag[i] == tag) {
        kind = bc->kind[i];
        adiab = bc->adiabatic ? bc->adiabatic[i] : 0;
        return true;
      }
    return false;
  };

  // ---- vertex order: Hilbert curve over the bounding box
  double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
  for (int i = 0; i < nv; ++i) {
    xmin = std::min(xmin, m.coords[2 * i]); xmax = std::max(xmax, m.coords[2 * i]);
    ymin = std::min(ymin, m.coords[2 * i + 1]); ymax = std::max(ymax, m.coords[2 * i + 1]);
  }
  double span = std::max(xmax - xmin, ymax - ymin);
  if (!(span > 0.0)) span = 1.0;
  std::vector<uint64_t> key(nv);
  for (int i = 0; i < nv; ++i) {
    double fx = (m.coords[2 * i] - xmin) / span, fy = (m.coords[2 * i + 1] - ymin) / span;
    uint32_t ix = (uint32_t)std::min(65535.0, std::max(0.0, std::floor(fx * 65535.0)));
    uint32_t iy = (uint32_t)std::min(65535.0, std::max(0.0, std::floor(fy * 65535.0)));
    key[i] = hilbert_index(ix, iy);
  }
  L.nv = nv;
  L.old_of_new.resize(nv);
  std::iota(L.old_of_new.begin(), L.old_of_new.end(), 0);
  std::stable_sort(L.old_of_new.begin(), L.old_of_new.end(), [&](int a, int b) { return key[a] < key[b]; });
  L.new_of_old.assign(nv, 0);
  for (int i = 0; i < nv; ++i) L.new_of_old[L.old_of_new[i]] = i;
  const std::vector<int>& N = L.new_of_old;

  L.axi = axi;
  if (axi) {
    L.v_r.resize(nv);
    for (int i = 0; i < nv; ++i) L.v_r[i] = m.vertex_radius[L.old_of_new[i]];
  }
  L.dcarea.resize(nv); L.inv6mc.resize(nv); L.pweight.resize(nv); L.x.resize(nv); L.y.resize(nv);
  for (int i = 0; i < nv; ++i) {
    int o = L.old_of_new[i];
    L.dcarea[i] = m.dcarea[o];
    L.inv6mc[i] = 1.0 / (6.0 * m.mcarea[o]);          // src/fv.cc:1040
    L.x[i] = m.coords[2 * o];
    L.y[i] = m.coords[2 * o + 1];
    // weight in norms / integrals: 1/|P_i| for periodic vertices (src/grid_preproc.cc:1037-1052)
    L.pweight[i] = set_of[o] >= 0 ? 1.0 / ((double)(m.periodic_offsets[set_of[o] + 1] - m.periodic_offsets[set_of[o]]) * 1.0)
                                  : 1.0 / 1.0;
  }

  // ---- edges: every reference face, plus each primal edge whose dual face the
  // reference dropped for zero measure (Voronoi duals, src/grid_preproc.cc:633-647):
  // those carry no flux (zero normal) but their P1 weights belong to the vertex
  // gradients, which the reference forms cell by cell
  std::vector<int> fvx(m.face_vertex, m.face_vertex + 2 * (size_t)nf);
  std::vector<double> fnrm(m.face_normal, m.face_normal + 2 * (size_t)nf);
  std::vector<int> flc(m.face_lcell, m.face_lcell + nf), frc(m.face_rcell, m.face_rcell + nf);
  {
    auto pkey = [](int a, int b) { return ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b); };
    std::unordered_map<uint64_t, int> seen;
    seen.reserve(2 * (size_t)nf);
    for (int f = 0; f < nf; ++f) seen.emplace(pkey(m.face_vertex[2 * f], m.face_vertex[2 * f + 1]), -1);
    for (int c = 0; c < nc; ++c)
      for (int k = 0; k < 3; ++k) {
        const int a = m.cell_vertex[3 * c + k], b = m.cell_vertex[3 * c + (k + 1) % 3];
        auto it = seen.find(pkey(a, b));
        if (it == seen.end()) {
          seen.emplace(pkey(a, b), (int)flc.size());
          fvx.push_back(a); fvx.push_back(b);
          fnrm.push_back(0.0); fnrm.push_back(0.0);
          flc.push_back(c); frc.push_back(-1);
        } else if (it->second >= 0) {
          frc[it->second] = c;
        }
      }
  }
  const int nfa = (int)flc.size();
  std::vector<int> eorder(nfa);
  std::iota(eorder.begin(), eorder.end(), 0);
  auto lo = [&](int f) { return std::min(N[fvx[2 * f]], N[fvx[2 * f + 1]]); };
  auto hi = [&](int f) { return std::max(N[fvx[2 * f]], N[fvx[2 * f + 1]]); };
  std::stable_sort(eorder.begin(), eorder.end(), [&](int a, int b) {
    int la = lo(a), lb = lo(b);
    if (la != lb) return la < lb;
    return hi(a) < hi(b);
  });
  L.ne = nfa;
  L.e_a.resize(nfa); L.e_b.resize(nfa); L.e_face.resize(nfa);
  L.e_nx.resize(nfa); L.e_ny.resize(nfa); L.e_dx.resize(nfa); L.e_dy.resize(nfa);
  L.e_g0x.assign(nfa, 0.0); L.e_g0y.assign(nfa, 0.0); L.e_g1x.assign(nfa, 0.0); L.e_g1y.assign(nfa, 0.0);
  for (int e = 0; e < nfa; ++e) {
    int f = eorder[e];
    int va = fvx[2 * f], vb = fvx[2 * f + 1];
    L.e_face[e] = f;
    L.e_a[e] = N[va];
    L.e_b[e] = N[vb];
    L.e_nx[e] = fnrm[2 * f];
    L.e_ny[e] = fnrm[2 * f + 1];
    if (axi) L.e_r.push_back(f < nf ? m.face_radius[f] : 1.0);   // gradient-only edges carry no flux
    L.e_dx[e] = m.coords[2 * vb] - m.coords[2 * va];     // src/kepes_tecno_roe.cc:112
    L.e_dy[e] = m.coords[2 * vb + 1] - m.coords[2 * va + 1];
    // gradient weights: sum over the face's cells of the P1 normal of the other endpoint
    int cells[2] = {flc[f], frc[f]};
    for (int q = 0; q < 2; ++q) {
      int c = cells[q];
      if (c < 0) continue;
      int ka = -1, kb = -1;
      for (int k = 0; k < 3; ++k) {
        if (m.cell_vertex[3 * c + k] == va) ka = k;
        if (m.cell_vertex[3 * c + k] == vb) kb = k;
      }
      if (ka < 0 || kb < 0) return "face vertices are not vertices of its cell";
      L.e_g0x[e] += m.cell_normal[6 * c + 2 * kb];
      L.e_g0y[e] += m.cell_normal[6 * c + 2 * kb + 1];
      L.e_g1x[e] += m.cell_normal[6 * c + 2 * ka];
      L.e_g1y[e] += m.cell_normal[6 * c + 2 * ka + 1];
    }
  }

  // members of the periodic group of a (reference) vertex, in set order
  auto group = [&](int o, std::vector<int>& g) {
    g.clear();
    if (set_of[o] < 0) { g.push_back(o); return; }
    for (int j = m.periodic_offsets[set_of[o]]; j < m.periodic_offsets[set_of[o] + 1]; ++j)
      g.push_back(m.periodic_members[j]);
  };

  // per reference vertex incident edges (in edge order)
  std::vector<std::vector<int>> inc(nv);
  for (int e = 0; e < nfa; ++e) {
    inc[fvx[2 * L.e_face[e]]].push_back(e << 1);
    inc[fvx[2 * L.e_face[e] + 1]].push_back((e << 1) | 1);
  }
  L.ce_off.assign(nv + 1, 0);
  std::vector<int> g;
  for (int i = 0; i < nv; ++i) {
    group(L.old_of_new[i], g);
    size_t cnt = 0;
    for (int o : g) cnt += inc[o].size();
    L.ce_off[i + 1] = L.ce_off[i] + (int)cnt;
  }
  L.ce_ent.resize(L.ce_off[nv]);
  for (int i = 0; i < nv; ++i) {
    group(L.old_of_new[i], g);
    int p = L.ce_off[i];
    for (int o : g)
      for (int x : inc[o]) L.ce_ent[p++] = x;
  }

  // ---- non-periodic boundary faces
  std::vector<int> dev_bface(nbf, -1);
  for (int b = 0; b < nbf; ++b) {
    int kind, adiab;
    bc_of(m.bface_type[b], kind, adiab);
    if (m.bface_periodic[b]) continue;
    if (kind == 0) {
      std::snprintf(buf, sizeof(buf), "no boundary condition for boundary tag %d", m.bface_type[b]);
      return buf;
    }
    if (kind == 7) continue;  // periodic tag: treated like the reference (no flux, no correction)
    dev_bface[b] = L.nb++;
  }
  const int nb = L.nb;
  L.b_v0.resize(nb); L.b_v1.resize(nb); L.b_kind.resize(nb); L.b_adiab.resize(nb); L.b_cell.resize(nb);
  L.b_nx.resize(nb); L.b_ny.resize(nb); L.b_val.assign((size_t)nb * 10, 0.0);
  L.bf_face_nx.resize(nb); L.bf_face_ny.resize(nb); L.bf_face_v0.resize(nb); L.bf_face_v1.resize(nb);
  std::vector<int> ref_bface_of_dev(nb);
  L.rb_type.assign(m.bface_type, m.bface_type + nbf);
  L.rb_v0.resize(nbf);
  L.rb_dev.resize(nbf);
  for (int b = 0; b < nbf; ++b) { L.rb_v0[b] = m.bface_vertex[2 * b]; L.rb_dev[b] = dev_bface[b]; }
  for (int b = 0; b < nbf; ++b) {
    int d = dev_bface[b];
    if (d < 0) continue;
    ref_bface_of_dev[d] = b;
    int kind, adiab;
    bc_of(m.bface_type[b], kind, adiab);
    L.b_v0[d] = N[m.bface_vertex[2 * b]];
    L.b_v1[d] = N[m.bface_vertex[2 * b + 1]];
    L.b_kind[d] = kind;
    L.b_adiab[d] = adiab;
    L.b_cell[d] = m.bface_lcell[b];
    L.b_nx[d] = m.bface_normal[2 * b];
    L.b_ny[d] = m.bface_normal[2 * b + 1];
    if (bc && bc->bface_values)
      for (int q = 0; q < 10; ++q) L.b_val[(size_t)d * 10 + q] = bc->bface_values[(size_t)b * 10 + q];
    L.bf_face_nx[d] = m.face_normal[2 * b];
    L.bf_face_ny[d] = m.face_normal[2 * b + 1];
    L.bf_face_v0[d] = N[m.face_vertex[2 * b]];
    L.bf_face_v1[d] = N[m.face_vertex[2 * b + 1]];
  }

  // cells' non-periodic boundary faces (left-cell relation, face order)
  std::vector<std::vector<int>> cell_bf(nc);
  for (int d = 0; d < nb; ++d) cell_bf[L.b_cell[d]].push_back(d);

  // ---- viscous units
  std::vector<std::vector<int>> inc_b(nv);   // per reference vertex: tagged boundary entries
  for (int d = 0; d < nb; ++d) {
    int b = ref_bface_of_dev[d];
    inc_b[m.bface_vertex[2 * b]].push_back(((2 * d + 0) << 2) | 0);
    inc_b[m.bface_vertex[2 * b + 1]].push_back(((2 * d + 1) << 2) | 0);
  }
  for (int c = 0; c < nc; ++c)
    for (int d : cell_bf[c])
      for (int k = 0; k < 3; ++k) inc_b[m.cell_vertex[3 * c + k]].push_back((d << 2) | 1);
  if (need_viscous) {
    // cell face slots in ascending face order (src/grid_preproc.cc:528-551)
    std::vector<int> cface(3 * (size_t)nc, -1);
    for (int f = 0; f < nf; ++f) {
      int c = m.face_lcell[f], j = 0;
      while (cface[3 * c + j] != -1) ++j;
      cface[3 * c + j] = f;
      c = m.face_rcell[f];
      if (c >= 0) { j = 0; while (cface[3 * c + j] != -1) ++j; cface[3 * c + j] = f; }
    }
    L.c_v.resize(3 * (size_t)nc); L.c_n.resize(6 * (size_t)nc); L.c_inv2a.resize(nc);
    L.c_bf_off.assign(nc + 1, 0); L.c_nbr_off.assign(nc + 1, 0);
    for (int c = 0; c < nc; ++c) {
      for (int k = 0; k < 3; ++k) L.c_v[3 * c + k] = N[m.cell_vertex[3 * c + k]];
      for (int k = 0; k < 6; ++k) L.c_n[6 * c + k] = m.cell_normal[6 * c + k];
      L.c_inv2a[c] = 1.0 / (2.0 * m.cell_area[c]);                    // src/fv.cc:1051
      L.c_bf_off[c + 1] = L.c_bf_off[c] + (int)cell_bf[c].size();
      for (int d : cell_bf[c]) L.c_bf.push_back(d);
      int cnt = 0;
      for (int j = 0; j < 3; ++j) {                                     // nbr_bface (src/grid_preproc.cc:811-832)
        int f = cface[3 * c + j];
        if (f >= 0 && f < nbf && dev_bface[f] >= 0) { L.c_nbr.push_back(dev_bface[f]); ++cnt; }
      }
      L.c_nbr_off[c + 1] = L.c_nbr_off[c] + cnt;
    }
    // units: interior cells first (cell order), then one per boundary face (face order)
    for (int c = 0; c < nc; ++c)
      if (L.c_nbr_off[c + 1] == L.c_nbr_off[c]) L.u_cell.push_back(c);
    L.n_int_cells = (int)L.u_cell.size();
    for (int d = 0; d < nb; ++d) L.u_cell.push_back(L.b_cell[d]);
    L.nvu = (int)L.u_cell.size();
    if (axi)
      for (int u = 0; u < L.nvu; ++u) L.u_r.push_back(m.cell_radius[L.u_cell[u]]);
    for (int u = 0; u < L.nvu; ++u) {
      int c = L.u_cell[u];
      for (int k = 0; k < 3; ++k) inc_b[m.cell_vertex[3 * c + k]].push_back(((3 * u + k) << 2) | 2);
      if (u >= L.n_int_cells) {
        int d = u - L.n_int_cells;
        int b = ref_bface_of_dev[d];
        inc_b[m.bface_vertex[2 * b]].push_back((d << 2) | 3);
        inc_b[m.bface_vertex[2 * b + 1]].push_back((d << 2) | 3);
      }
    }
  }
  L.cb_off.assign(nv + 1, 0);
  for (int i = 0; i < nv; ++i) {
    group(L.old_of_new[i], g);
    size_t cnt = 0;
    for (int o : g) cnt += inc_b[o].size();
    L.cb_off[i + 1] = L.cb_off[i] + (int)cnt;
  }
  L.cb_ent.resize(L.cb_off[nv]);
  for (int i = 0; i < nv; ++i) {
    group(L.old_of_new[i], g);
    int p = L.cb_off[i];
    for (int o : g)
      for (int x : inc_b[o]) L.cb_ent[p++] = x;
  }
  // the fixed-order gather relies on indices fitting the entry encodings
  if ((long long)nf * 2 >= (1LL << 31) || (long long)L.nvu * 3 >= (1LL << 29) || (long long)nb * 2 >= (1LL << 29))
    return "mesh too large for 32-bit gather entries";
  return "";
}

std::string build_tiles(HostLayout& L, int max_owned, int max_local, int max_edges) {
  const int nv = L.nv;
  const int n_own = L.n_owned >= 0 ? L.n_owned : nv;   // tiles cover the owned vertices only
  if (max_owned <= 0 || max_local > 65535 || max_edges > 32767) return "bad tile limits";
  L.t_vbeg.clear(); L.t_loff.assign(1, 0); L.t_eoff.assign(1, 0); L.lv.clear();
  L.te_ab.clear(); L.te_nx.clear(); L.te_ny.clear();
  L.te_g0x.clear(); L.te_g0y.clear(); L.te_g1x.clear(); L.te_g1y.clear();
  L.te_ux.clear(); L.te_uy.clear(); L.te_ar.clear(); L.te_r.clear();
  L.cv_off.assign(nv + 1, 0);
  L.cv_ent.clear();
  L.lmax = L.emax = L.tmax = L.cmax = 0;
  // scratch maps global id -> tile-local id, reset per tile
  std::vector<int> vloc(nv, -1), eloc(L.ne, -1);
  std::vector<int> tv, te;  // current tile's local vertices / edges (global ids)
  int v = 0;
  while (v < n_own) {
    int vb = v;
    tv.clear();
    te.clear();
    // greedily add owned vertices while the neighbourhood fits
    int nown = 0;
    while (v < n_own && nown < max_owned) {
      // tentative: count new edges and new local vertices of vertex v
      int add_e = 0, add_v = (vloc[v] < 0) ? 1 : 0;
      std::vector<int> new_halo;
      for (int j = L.ce_off[v]; j < L.ce_off[v + 1]; ++j) {
        int e = L.ce_ent[j] >> 1;
        if (eloc[e] >= 0) continue;
        ++add_e;
        for (int x : {L.e_a[e], L.e_b[e]})
          if (vloc[x] < 0 && x != v) {
            bool seen = false;
            for (int y : new_halo) seen |= (y == x);
            if (!seen) { new_halo.push_back(x); ++add_v; }
          }
      }
      if (nown > 0 && ((int)tv.size() + add_v > max_local || (int)te.size() + add_e > max_edges)) break;
      // commit: owned vertices must occupy local ids 0..nown-1, so an owned
      // vertex that is already a halo entry of this tile is moved to the front later
      if (vloc[v] < 0) { vloc[v] = (int)tv.size(); tv.push_back(v); }
      for (int j = L.ce_off[v]; j < L.ce_off[v + 1]; ++j) {
        int e = L.ce_ent[j] >> 1;
        if (eloc[e] >= 0) continue;
        eloc[e] = (int)te.size();
        te.push_back(e);
        for (int x : {L.e_a[e], L.e_b[e]})
          if (vloc[x] < 0) { vloc[x] = (int)tv.size(); tv.push_back(x); }
      }
      ++nown;
      ++v;
    }
    // reorder local vertices: owned [vb, v) first, in order, then the halo in first-seen order
    std::vector<int> order;
    order.reserve(tv.size());
    for (int x = vb; x < v; ++x) order.push_back(x);
    for (int x : tv)
      if (x < vb || x >= v) order.push_back(x);
    for (size_t i = 0; i < order.size(); ++i) vloc[order[i]] = (int)i;
    if ((int)order.size() > 65535 || (int)te.size() > 32767) return "tile neighbourhood too large";
    L.t_vbeg.push_back(vb);
    for (int x : order) L.lv.push_back(x);
    L.t_loff.push_back((int)L.lv.size());
    for (int e : te) {
      L.te_ab.push_back((uint32_t)vloc[L.e_a[e]] | ((uint32_t)vloc[L.e_b[e]] << 16));
      L.te_nx.push_back(L.e_nx[e]); L.te_ny.push_back(L.e_ny[e]);
      L.te_g0x.push_back(L.e_g0x[e]); L.te_g0y.push_back(L.e_g0y[e]);
      L.te_g1x.push_back(L.e_g1x[e]); L.te_g1y.push_back(L.e_g1y[e]);
      // src/material.cc:69 area = normal.norm(); src/kepec.cc:18 unit = normal * (1/area);
      // a gradient-only edge (zero normal) gets a zero unit normal, so its flux is zero
      double area = std::sqrt(L.e_nx[e] * L.e_nx[e] + L.e_ny[e] * L.e_ny[e] + 0.0 * 0.0);
      double ia = area > 0.0 ? 1.0 / area : 0.0;
      L.te_ux.push_back(L.e_nx[e] * ia);
      L.te_uy.push_back(L.e_ny[e] * ia);
      L.te_ar.push_back(area);
      if (L.axi) L.te_r.push_back(L.e_r[e]);
    }
    L.t_eoff.push_back((int)L.te_ab.size());
    for (int x = vb; x < v; ++x) {
      for (int j = L.ce_off[x]; j < L.ce_off[x + 1]; ++j) {
        int ent = L.ce_ent[j];
        L.cv_ent.push_back((uint16_t)((eloc[ent >> 1] << 1) | (ent & 1)));
      }
      L.cv_off[x + 1] = (int)L.cv_ent.size();
    }
    L.cmax = std::max(L.cmax, L.cv_off[v] - L.cv_off[vb] + 1);   // +1: staging starts on an even entry
    L.lmax = std::max(L.lmax, (int)order.size());
    L.emax = std::max(L.emax, (int)te.size());
    L.tmax = std::max(L.tmax, v - vb);
    for (int x : order) vloc[x] = -1;
    for (int e : te) eloc[e] = -1;
  }
  L.t_vbeg.push_back(n_own);
  for (int x = n_own; x < nv; ++x) L.cv_off[x + 1] = L.cv_off[x];   // ghosts: empty lists
  L.ntiles = (int)L.t_vbeg.size() - 1;
  if (L.cv_ent.size() & 1) L.cv_ent.push_back(0);   // the lists are staged in whole 4-byte words
  return "";
}

namespace {

// Device ids a vertex's gather lists read: edge endpoints (periodic partners'
// edges included) and the vertices of its boundary faces.
template <class F>
void for_each_reach(const HostLayout& G, int v, F&& f) {
  for (int j = G.ce_off[v]; j < G.ce_off[v + 1]; ++j) {
    const int e = G.ce_ent[j] >> 1;
    f(G.e_a[e]);
    f(G.e_b[e]);
  }
  for (int j = G.cb_off[v]; j < G.cb_off[v + 1]; ++j) {
    const int ent = G.cb_ent[j], type = ent & 3, idx = ent >> 2;
    if (type == 2) {   // a viscous unit: the vertices of its cell (and of its cell's boundary faces)
      const int c = G.u_cell[idx / 3];
      for (int k = 0; k < 3; ++k) f(G.c_v[3 * (size_t)c + k]);
      continue;
    }
    const int d = type == 0 ? idx >> 1 : idx;
    f(G.b_v0[d]); f(G.b_v1[d]);
    if (G.nvu > 0) {   // the face's boundary unit reads its cell
      const int c = G.b_cell[d];
      for (int k = 0; k < 3; ++k) f(G.c_v[3 * (size_t)c + k]);
    }
  }
}

int owner_of(const std::vector<int>& v0, int v) {
  return (int)(std::upper_bound(v0.begin(), v0.end(), v) - v0.begin()) - 1;
}

// Ghosts of partition q: vertices outside its range that its owned vertices reach.
std::vector<int> ghosts_of(const HostLayout& G, const std::vector<int>& v0, int q) {
  std::vector<int> g;
  for (int v = v0[q]; v < v0[q + 1]; ++v)
    for_each_reach(G, v, [&](int x) { if (x < v0[q] || x >= v0[q + 1]) g.push_back(x); });
  std::sort(g.begin(), g.end());
  g.erase(std::unique(g.begin(), g.end()), g.end());
  return g;
}

}  // namespace

std::string plan_partition(const HostLayout& G, int n_parts, int part, PartPlan& P) {
  if (n_parts < 1 || part < 0 || part >= n_parts) return "partition index out of range";
  if (n_parts > G.nv) return "more partitions than vertices";
  P = PartPlan();
  P.n_parts = n_parts;
  P.part = part;
  P.v0.resize(n_parts + 1);
  for (int q = 0; q <= n_parts; ++q) P.v0[q] = (int)((long long)q * G.nv / n_parts);
  const int a = P.v0[part], b = P.v0[part + 1];
  P.n_owned = b - a;
  const std::vector<int> mine = ghosts_of(G, P.v0, part);
  P.local.resize(P.n_owned);
  for (int v = a; v < b; ++v) P.local[v - a] = v;
  P.local.insert(P.local.end(), mine.begin(), mine.end());
  // receive lists: my ghosts grouped by owner (ascending device id within each)
  P.recv_off.assign(n_parts + 1, 0);
  {
    std::vector<std::vector<int>> by(n_parts);
    for (size_t i = 0; i < mine.size(); ++i) by[owner_of(P.v0, mine[i])].push_back(P.n_owned + (int)i);
    for (int q = 0; q < n_parts; ++q) {
      P.recv_idx.insert(P.recv_idx.end(), by[q].begin(), by[q].end());
      P.recv_off[q + 1] = (int)P.recv_idx.size();
    }
  }
  // send lists: for each peer, my owned vertices among its ghosts (ascending)
  P.send_off.assign(n_parts + 1, 0);
  for (int q = 0; q < n_parts; ++q) {
    if (q != part)
      for (int x : ghosts_of(G, P.v0, q))
        if (x >= a && x < b) P.send_idx.push_back(x - a);
    P.send_off[q + 1] = (int)P.send_idx.size();
  }
  return "";
}

std::string restrict_layout(const HostLayout& G, const PartPlan& P, HostLayout& L) {
  const int nloc = (int)P.local.size(), nown = P.n_owned;
  L = HostLayout();
  L.nv = nloc;
  L.n_owned = nown;
  std::vector<int> lid(G.nv, -1);
  for (int i = 0; i < nloc; ++i) lid[P.local[i]] = i;
  L.old_of_new.resize(nloc);
  L.axi = G.axi;
  for (int i = 0; i < nloc; ++i) {
    const int g = P.local[i];
    L.old_of_new[i] = G.old_of_new[g];
    L.dcarea.push_back(G.dcarea[g]); L.inv6mc.push_back(G.inv6mc[g]); L.pweight.push_back(G.pweight[g]);
    L.x.push_back(G.x[g]); L.y.push_back(G.y[g]);
    if (G.axi) L.v_r.push_back(G.v_r[g]);
  }
  // edges, boundary faces and interior viscous units the owned vertices' lists use,
  // in the global order
  std::vector<int> edges, faces, iunits;
  for (int v = P.v0[P.part]; v < P.v0[P.part + 1]; ++v) {
    for (int j = G.ce_off[v]; j < G.ce_off[v + 1]; ++j) edges.push_back(G.ce_ent[j] >> 1);
    for (int j = G.cb_off[v]; j < G.cb_off[v + 1]; ++j) {
      const int ent = G.cb_ent[j], type = ent & 3, idx = ent >> 2;
      if (type == 2) {
        const int u = idx / 3;
        if (u < G.n_int_cells) iunits.push_back(u);
        else faces.push_back(u - G.n_int_cells);   // a boundary unit belongs to its face
      } else {
        faces.push_back(type == 0 ? idx >> 1 : idx);
      }
    }
  }
  if (G.nvu > 0) {
    // every local boundary face gets its boundary unit, which reads the boundary faces of
    // the face's cell (its gradient corrections and boundary states): those join the set
    const size_t n0 = faces.size();
    for (size_t i = 0; i < n0; ++i) {
      const int c = G.b_cell[faces[i]];
      for (int j = G.c_bf_off[c]; j < G.c_bf_off[c + 1]; ++j) faces.push_back(G.c_bf[j]);
      for (int j = G.c_nbr_off[c]; j < G.c_nbr_off[c + 1]; ++j) faces.push_back(G.c_nbr[j]);
    }
  }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  std::sort(faces.begin(), faces.end());
  faces.erase(std::unique(faces.begin(), faces.end()), faces.end());
  std::sort(iunits.begin(), iunits.end());
  iunits.erase(std::unique(iunits.begin(), iunits.end()), iunits.end());
  std::vector<int> elid(G.ne, -1), blid(G.nb, -1);
  L.ne = (int)edges.size();
  for (int i = 0; i < L.ne; ++i) {
    const int e = edges[i];
    elid[e] = i;
    if (lid[G.e_a[e]] < 0 || lid[G.e_b[e]] < 0) return "partition edge endpoint is not local";
    L.e_a.push_back(lid[G.e_a[e]]); L.e_b.push_back(lid[G.e_b[e]]); L.e_face.push_back(G.e_face[e]);
    L.e_nx.push_back(G.e_nx[e]); L.e_ny.push_back(G.e_ny[e]); L.e_dx.push_back(G.e_dx[e]); L.e_dy.push_back(G.e_dy[e]);
    L.e_g0x.push_back(G.e_g0x[e]); L.e_g0y.push_back(G.e_g0y[e]);
    L.e_g1x.push_back(G.e_g1x[e]); L.e_g1y.push_back(G.e_g1y[e]);
    if (G.axi) L.e_r.push_back(G.e_r[e]);
  }
  L.nb = (int)faces.size();
  for (int i = 0; i < L.nb; ++i) {
    const int d = faces[i];
    blid[d] = i;
    if (lid[G.b_v0[d]] < 0 || lid[G.b_v1[d]] < 0) return "partition boundary-face vertex is not local";
    L.b_v0.push_back(lid[G.b_v0[d]]); L.b_v1.push_back(lid[G.b_v1[d]]);
    L.b_kind.push_back(G.b_kind[d]); L.b_adiab.push_back(G.b_adiab[d]); L.b_cell.push_back(G.b_cell[d]);
    L.b_nx.push_back(G.b_nx[d]); L.b_ny.push_back(G.b_ny[d]);
    L.b_val.insert(L.b_val.end(), G.b_val.begin() + (size_t)d * 10, G.b_val.begin() + (size_t)d * 10 + 10);
    L.bf_face_nx.push_back(G.bf_face_nx[d]); L.bf_face_ny.push_back(G.bf_face_ny[d]);
    L.bf_face_v0.push_back(std::max(0, lid[G.bf_face_v0[d]])); L.bf_face_v1.push_back(std::max(0, lid[G.bf_face_v1[d]]));
  }
  // viscous units: the interior units the owned vertices gather, then one boundary unit per
  // local boundary face in local face order (the device's unit numbering); their cells
  // with local vertex and face ids
  std::vector<int> ulid(G.nvu, -1);
  if (G.nvu > 0) {
    std::vector<int> units = iunits;
    for (int d : faces) units.push_back(G.n_int_cells + d);
    L.n_int_cells = (int)iunits.size();
    L.nvu = (int)units.size();
    std::vector<int> clid;
    std::vector<int> cells;
    for (int u : units) cells.push_back(G.u_cell[u]);
    std::vector<int> ucell_sorted = cells;
    std::sort(ucell_sorted.begin(), ucell_sorted.end());
    ucell_sorted.erase(std::unique(ucell_sorted.begin(), ucell_sorted.end()), ucell_sorted.end());
    const int ncl = (int)ucell_sorted.size();
    L.c_bf_off.assign(ncl + 1, 0);
    L.c_nbr_off.assign(ncl + 1, 0);
    for (int i = 0; i < ncl; ++i) {
      const int c = ucell_sorted[i];
      for (int k = 0; k < 3; ++k) {
        const int x = lid[G.c_v[3 * (size_t)c + k]];
        if (x < 0) return "partition viscous-cell vertex is not local";
        L.c_v.push_back(x);
      }
      for (int k = 0; k < 6; ++k) L.c_n.push_back(G.c_n[6 * (size_t)c + k]);
      L.c_inv2a.push_back(G.c_inv2a[c]);
      for (int j = G.c_bf_off[c]; j < G.c_bf_off[c + 1]; ++j) {
        if (blid[G.c_bf[j]] < 0) return "partition viscous-cell boundary face is not local";
        L.c_bf.push_back(blid[G.c_bf[j]]);
      }
      for (int j = G.c_nbr_off[c]; j < G.c_nbr_off[c + 1]; ++j) {
        if (blid[G.c_nbr[j]] < 0) return "partition viscous-cell boundary face is not local";
        L.c_nbr.push_back(blid[G.c_nbr[j]]);
      }
      L.c_bf_off[i + 1] = (int)L.c_bf.size();
      L.c_nbr_off[i + 1] = (int)L.c_nbr.size();
    }
    for (size_t i = 0; i < units.size(); ++i) {
      ulid[units[i]] = (int)i;
      const int c = (int)(std::lower_bound(ucell_sorted.begin(), ucell_sorted.end(), cells[i]) - ucell_sorted.begin());
      L.u_cell.push_back(c);
      if (G.axi) L.u_r.push_back(G.u_r[units[i]]);
    }
    for (int d : faces)
      if (lid[G.bf_face_v0[d]] < 0 || lid[G.bf_face_v1[d]] < 0) return "partition viscous boundary vertex is not local";
    for (int i = 0; i < L.nb; ++i)   // the boundary faces' cells in the local cell numbering
      L.b_cell[i] = (int)(std::lower_bound(ucell_sorted.begin(), ucell_sorted.end(), G.b_cell[faces[i]]) -
                          ucell_sorted.begin());
  }
  // owned vertices keep their lists, entry for entry; ghosts have none
  L.ce_off.assign(nloc + 1, 0);
  L.cb_off.assign(nloc + 1, 0);
  for (int i = 0; i < nown; ++i) {
    const int v = P.local[i];
    for (int j = G.ce_off[v]; j < G.ce_off[v + 1]; ++j) {
      const int ent = G.ce_ent[j];
      L.ce_ent.push_back((elid[ent >> 1] << 1) | (ent & 1));
    }
    for (int j = G.cb_off[v]; j < G.cb_off[v + 1]; ++j) {
      const int ent = G.cb_ent[j], type = ent & 3, idx = ent >> 2;
      const int nidx = type == 0 ? ((blid[idx >> 1] << 1) | (idx & 1))
                       : type == 2 ? 3 * ulid[idx / 3] + idx % 3 : blid[idx];
      L.cb_ent.push_back((nidx << 2) | type);
    }
    L.ce_off[i + 1] = (int)L.ce_ent.size();
    L.cb_off[i + 1] = (int)L.cb_ent.size();
  }
  for (int i = nown; i < nloc; ++i) { L.ce_off[i + 1] = L.ce_off[i]; L.cb_off[i + 1] = L.cb_off[i]; }
  return "";
}

std::string force_faces(const HostLayout& L, int n_forces, const int* n_tags, const int* tags, std::vector<int>& rec4,
                        std::vector<int>& off) {
  const int nbf = (int)L.rb_type.size();
  rec4.clear();
  off.assign(1, 0);
  const int* t = tags;
  for (int f = 0; f < n_forces; ++f) {
    if (n_tags[f] < 1) return "a force needs at least one face tag (src/parameter.cc:652)";
    // the condition the reference applies on every face of force f is that of bface[f] (src/force.cc:144-150)
    int dq = -1, k0 = 0, k1 = 0;
    for (int b = 0; b < nbf; ++b) {
      bool mine = false;
      for (int q = 0; q < n_tags[f]; ++q) mine = mine || L.rb_type[b] == t[q];
      if (!mine) continue;
      if (L.rb_dev[b] < 0) return "force faces must not be periodic";
      if (f < nbf) {
        dq = L.rb_dev[f];
        const int dv0 = L.b_v0[L.rb_dev[b]], dv1 = L.b_v1[L.rb_dev[b]];
        const int q0 = L.new_of_old[L.rb_v0[f]];
        k0 = (q0 == dv0) ? 0 : 1;   // value slot: vertex 0 of bface[f] or not (src/bc.h:568-654 via the table)
        k1 = (q0 == dv1) ? 0 : 1;
      }
      rec4.insert(rec4.end(), {L.rb_dev[b], dq, k0, k1});
    }
    if ((int)rec4.size() / 4 == off.back()) return "a force tag matches no boundary face";
    off.push_back((int)rec4.size() / 4);
    t += n_tags[f];
  }
  return "";
}

}  // namespace tg
