// tg_mesh.h -- host-side construction of the device mesh layout.
//
// Input: the reference's Grid after preproc (tg_mesh, reference numbering).
// Output: flat arrays in the device numbering (vertices reordered along a
// Hilbert curve, edges sorted by their lower vertex) plus the per-vertex
// gather lists that make every accumulation deterministic.
//
// Periodic vertices are kept as separate degrees of freedom, as the reference
// stores them.  The reference sums residual, gradient and dt contributions
// over each periodic set and copies the sum back
// (src/reduce_residual_periodic.cc:18-31,122-130, src/reduce_gradient_periodic.cc,
// src/reduce_dt_periodic.cc); here every member's gather list is the union of
// the lists of all members of its set, in a fixed order, so each copy computes
// that same sum itself in one pass and all copies end bitwise equal.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/tensum_gpu.h"

namespace tg {

struct HostLayout {
  int nv = 0;          // vertices (reference n_vertex, periodic copies included)
  int ne = 0;          // edges    (reference faces, boundary and periodic faces included)
  int nb = 0;          // non-periodic boundary faces
  int nvu = 0;         // viscous units: interior cells + one per non-periodic boundary face
  std::vector<int> new_of_old, old_of_new;
  // vertices (device order)
  std::vector<double> dcarea, inv6mc, pweight, x, y;
  // axisymmetric radii (src/grid_preproc.cc:750-777; empty when planar): per vertex,
  // per edge (its reference face's radius) and per viscous unit (its cell's radius)
  bool axi = false;
  std::vector<double> v_r, e_r, u_r;
  // edges
  std::vector<int> e_a, e_b, e_face;
  std::vector<double> e_nx, e_ny, e_dx, e_dy, e_g0x, e_g0y, e_g1x, e_g1y;
  // per-vertex edge gather: entry = (edge << 1) | side   (side 1 = vertex is endpoint b)
  std::vector<int> ce_off, ce_ent;
  // non-periodic boundary faces
  std::vector<int> b_v0, b_v1, b_kind, b_adiab, b_cell;
  std::vector<double> b_nx, b_ny, b_val;  // b_val: nb*2*5 (T,u,v,w,p) at vertex 0 / 1
  // every reference boundary face: its tag, vertex 0 (reference numbering) and
  // its device index (-1 for periodic faces), for the force integrals
  std::vector<int> rb_type, rb_v0, rb_dev;
  // per-vertex boundary / viscous gather: entry = (index << 2) | type
  //   type 0: inviscid boundary flux (2*b + k)     type 1: gradient boundary correction (b)
  //   type 2: viscous unit contribution (3*u + k)  type 3: viscous boundary flux (b)
  std::vector<int> cb_off, cb_ent;
  // viscous units: u < n_int_cells -> interior cell; else boundary face (u - n_int_cells)
  int n_int_cells = 0;
  std::vector<int> u_cell;                 // cell id (device cell numbering) per unit
  std::vector<int> c_v;                    // 3 per cell (device vertex ids)
  std::vector<double> c_n;                 // 6 per cell: P1 normals
  std::vector<double> c_inv2a;             // 1/(2 area)
  std::vector<int> c_bf_off, c_bf;         // non-periodic boundary faces with this cell on their left, face order
  std::vector<int> c_nbr_off, c_nbr;       // the cell's non-periodic boundary faces in cell.face slot order
  std::vector<double> bf_face_nx, bf_face_ny;  // face-list normal of the boundary face (slip in viscous BC states)
  std::vector<int> bf_face_v0, bf_face_v1;     // face-list vertex order of the boundary face

  // ---- tiles: contiguous ranges of owned vertices with their edge neighbourhood
  // Tile t owns vertices [t_vbeg[t], t_vbeg[t+1]).  Its local vertex table
  // lv[t_loff[t] .. t_loff[t+1]) lists the owned vertices first, then every
  // other endpoint of the tile's edges.  Its edge list (te_*, t_eoff) holds
  // every edge incident to an owned vertex or to a periodic copy of one, with
  // endpoints as local indices (la | lb << 16).  cv_off/cv_ent is the owned
  // vertices' gather list in tile-local edge indices, (local_edge << 1) | side,
  // in exactly the order of ce_ent, so the tiled kernels sum in the same order.
  int ntiles = 0, lmax = 0, emax = 0, tmax = 0, cmax = 0;  // cmax: gather entries per tile
  // A partition's layout owns vertices [0, n_owned) only; the rest are ghosts that
  // the halo exchange fills (no tiles, no gather lists).  -1: every vertex is owned.
  int n_owned = -1;
  std::vector<int> t_vbeg, t_loff, t_eoff, lv;
  std::vector<uint32_t> te_ab;
  std::vector<double> te_nx, te_ny, te_g0x, te_g0y, te_g1x, te_g1y;
  std::vector<double> te_ux, te_uy, te_ar;   // n/|n| and |n|, as Material::num_flux forms them
  std::vector<double> te_r;                  // the edge's radius (axisymmetric runs)
  std::vector<int> cv_off;
  std::vector<uint16_t> cv_ent;
};

// Returns "" on success, else an error message.
std::string build_layout(const tg_mesh& m, const tg_bc_table* bc, bool need_viscous, HostLayout& out);

// Splits the (already built) layout into tiles of at most max_owned owned
// vertices, max_local local vertices and max_edges edges each.
std::string build_tiles(HostLayout& L, int max_owned, int max_local, int max_edges);

// Domain decomposition of one mesh into n_parts partitions: partition q owns the
// device-order vertex range [v0[q], v0[q+1]) and holds as ghosts every other vertex
// its owned vertices' gather lists reach (edge endpoints, periodic partners'
// neighbours, boundary-face vertices).  Each vertex is computed by its owner only,
// with the gather lists and their order unchanged, so a partitioned solve repeats
// the one-partition solve bit for bit; the reference's partitions instead sum
// partial residuals and gradients of shared vertices across processes
// (src/reduce_residual.cc:14-104, src/fv.cc:827-1030).
struct PartPlan {
  int n_parts = 0, part = 0;
  std::vector<int> v0;                 // n_parts + 1 range starts in the device order
  std::vector<int> local;              // device ids of this partition's vertices: owned, then ghosts ascending
  int n_owned = 0;
  // per peer q (offsets n_parts + 1): local ids of the owned vertices q holds as
  // ghosts, and local ids of the ghosts q owns, both in ascending device order, so
  // a sender's list and the receiver's list pair up entry by entry
  std::vector<int> send_off, send_idx, recv_off, recv_idx;
};

// Builds partition `part` of `n_parts` from the full layout.  A partition holds the
// viscous units its owned vertices gather (interior cells) and one per local boundary
// face, with their cells renumbered.  Strong-condition lists are not split (the caller
// refuses those runs).
std::string plan_partition(const HostLayout& G, int n_parts, int part, PartPlan& P);
std::string restrict_layout(const HostLayout& G, const PartPlan& P, HostLayout& out);

// Face records of compute_forces (src/force.cc:116-219) for n_forces force
// definitions (n_tags[f] face tags each, consecutive in `tags`): per face 4 ints
// (device face index, the device index of bface[f] whose condition the
// reference applies on every face of force f or -1, and the value slots that
// condition uses at the face's two vertices); off[f] .. off[f+1] index force f.
std::string force_faces(const HostLayout& L, int n_forces, const int* n_tags, const int* tags, std::vector<int>& rec4,
                        std::vector<int>& off);

}  // namespace tg
