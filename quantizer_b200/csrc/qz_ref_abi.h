/*
 * qz_ref_abi.h -- binary-compatible declarations of the two QUANTIZER data
 * structures the drop-in shim reads through pointers handed over by the host
 * program: struct cell_struct (headers/initialize_cell_struct.h:60-66) and
 * struct node (headers/initialize_node.h:63-216), with vtype = double
 * (headers/common.h:48-58, _VTYPE_ 2).
 *
 * Member order and types must match the reference's definitions exactly for
 * the shim to read the same memory; names are kept so that the shim reads
 * like the reference.  Comments state what each group holds.
 */
#ifndef QZ_REF_ABI_H
#define QZ_REF_ABI_H
#include <stdbool.h>

typedef double qz_vtype;

struct cell_struct {
    int *ptr_ptcl;      /* global indices of the cell's particles */
    int ptcl_cap;
    int ptcl_size;
    qz_vtype cell_mass;
};

struct node {
    int ID, lv;
    /* cell-status box: >=0 zone id, -1 refine, -3 in node, -4 not in node,
     * -5 outside the simulation, -6 periodic ghost */
    int *ptr_box, *ptr_box_old;
    int box_cap;
    int box_real_dim_x, box_real_dim_y, box_real_dim_z;
    int box_dim_x, box_dim_y, box_dim_z;
    int box_ts_x, box_ts_y, box_ts_z; /* cell index -> box index translation */
    int box_min_x, box_min_y, box_min_z;
    int box_max_x, box_max_y, box_max_z;
    bool box_check_fit;
    /* cells of the node */
    int *ptr_cell_idx_x, *ptr_cell_idx_y, *ptr_cell_idx_z, *ptr_box_idx;
    int cell_cap, cell_size;
    struct cell_struct *ptr_cell_struct, *ptr_cell_struct_old;
    int cell_struct_old_cap;
    qz_vtype node_mass;
    int no_ptcl_full_node, no_ptcl_outs_ref_zones;
    /* interior, boundary and simulation-boundary grid points */
    int *ptr_intr_grid_cell_idx_x, *ptr_intr_grid_cell_idx_y, *ptr_intr_grid_cell_idx_z;
    int *ptr_intr_box_grid_idx;
    int grid_intr_cap, grid_intr_size;
    int *ptr_bdry_grid_cell_idx_x, *ptr_bdry_grid_cell_idx_y, *ptr_bdry_grid_cell_idx_z;
    int *ptr_bdry_box_grid_idx;
    int grid_bdry_cap, grid_bdry_size;
    int *ptr_sim_bdry_grid_cell_idx_x, *ptr_sim_bdry_grid_cell_idx_y, *ptr_sim_bdry_grid_cell_idx_z;
    int *ptr_sim_bdry_box_grid_idx;
    int grid_sim_bdry_cap, grid_sim_bdry_size;
    /* grid fields, (box_real_dim + 1)^3 points */
    qz_vtype *ptr_pot, *ptr_pot_old, *ptr_ax, *ptr_ay, *ptr_az, *ptr_d;
    int grid_properties_cap;
    /* tree links */
    struct node **pptr_chn;
    struct node *ptr_pt;
    int chn_cap, chn_size;
    /* refinement bookkeeping */
    int *ptr_cell_ref;
    int cell_ref_cap, cell_ref_size;
    int **pptr_zones;
    int zones_cap, zones_size;
    int *ptr_zone_cap, *ptr_zone_size;
    int *ptr_aux_idx;
    int aux_idx_cap;
    bool *ptr_pbc_bool_bdry_anomalies_x, *ptr_pbc_bool_bdry_anomalies_y,
        *ptr_pbc_bool_bdry_anomalies_z;
    int pbc_bool_bdry_anomalies_cap;
    int *ptr_pbc_min_subzones_x, *ptr_pbc_min_subzones_y, *ptr_pbc_min_subzones_z;
    int *ptr_pbc_max_subzones_x, *ptr_pbc_max_subzones_y, *ptr_pbc_max_subzones_z;
    int pbc_subzones_cap, pbc_subzones_size;
    int *ptr_links_old_ord_old, *ptr_links_new_ord_new, *ptr_links_new_ord_old,
        *ptr_links_old_ord_new;
    int links_cap;
    /* simulation-boundary contact and periodic-boundary flags */
    bool sim_bdry_contact, sim_bdry_contact_x, sim_bdry_contact_y, sim_bdry_contact_z;
    bool pbc_crosses_sim_box_bdry, pbc_crosses_sim_box_bdry_x, pbc_crosses_sim_box_bdry_y,
        pbc_crosses_sim_box_bdry_z;
    bool pbc_crosses_whole_sim_box, pbc_crosses_whole_sim_box_x, pbc_crosses_whole_sim_box_y,
        pbc_crosses_whole_sim_box_z;
    bool pbc_correction_due_pbc_flag;
};

#endif
