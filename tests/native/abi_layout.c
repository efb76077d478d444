/* Prints the size and field offsets of every public struct of include/phmm_b200.h, fields in
 * declaration order, for tests/test_host.py to compare with the ctypes mirrors of the Python
 * package: "struct <name> <size>" then "field <name>.<field> <offset>". */
#include <stddef.h>
#include <stdio.h>

#include "../../include/phmm_b200.h"

#define S(T) printf("struct %s %zu\n", #T, sizeof(T))
#define F(T, f) printf("field %s.%s %zu\n", #T, #f, offsetof(T, f))

int main(void)
{
    S(phmm_config);
    F(phmm_config, device); F(phmm_config, use_cuda_graph); F(phmm_config, autotune); F(phmm_config, reserved0);
    F(phmm_config, hbm_budget_bytes); F(phmm_config, chunk_cells);
    S(phmm_batch);
    F(phmm_batch, n_regions); F(phmm_batch, n_haps); F(phmm_batch, n_reads); F(phmm_batch, hap_bases);
    F(phmm_batch, hap_off); F(phmm_batch, read_bases); F(phmm_batch, read_qual); F(phmm_batch, read_ins);
    F(phmm_batch, read_del); F(phmm_batch, read_gcp); F(phmm_batch, read_off);
    S(phmm_stats);
    F(phmm_stats, regions); F(phmm_stats, pairs); F(phmm_stats, cells); F(phmm_stats, pairs_f64);
    F(phmm_stats, work_items); F(phmm_stats, h2d_bytes); F(phmm_stats, d2h_bytes); F(phmm_stats, kernel_launches);
    F(phmm_stats, device_ms); F(phmm_stats, fp32_ms); F(phmm_stats, fp64_ms); F(phmm_stats, host_ms);
    S(phmm_tile_table);
    F(phmm_tile_table, rows_per_lane); F(phmm_tile_table, multi_stripe);
    S(phmm_tune_entry);
    F(phmm_tune_entry, mode); F(phmm_tune_entry, bucket); F(phmm_tune_entry, rows_per_lane);
    F(phmm_tune_entry, multi_stripe); F(phmm_tune_entry, chosen); F(phmm_tune_entry, reserved); F(phmm_tune_entry, gcups);
    S(phmm_tune_report);
    F(phmm_tune_report, n_entries); F(phmm_tune_report, reserved); F(phmm_tune_report, seconds);
    F(phmm_tune_report, entries);
    S(phmm_region_input);
    F(phmm_region_input, n_haps); F(phmm_region_input, hap_bases); F(phmm_region_input, hap_off);
    F(phmm_region_input, n_reads); F(phmm_region_input, read_bases); F(phmm_region_input, read_qual);
    F(phmm_region_input, read_off); F(phmm_region_input, mapq); F(phmm_region_input, min_quality_threshold);
    F(phmm_region_input, pcr_model);
    S(phmm_region_events);
    F(phmm_region_events, n_events); F(phmm_region_events, n_alleles); F(phmm_region_events, hap_allele);
    F(phmm_region_events, genotype_lk); F(phmm_region_events, best_genotype); F(phmm_region_events, allele_lk);
    S(phmm_region_realign);
    F(phmm_region_realign, hap_priority); F(phmm_region_realign, clip_left); F(phmm_region_realign, clip_right);
    F(phmm_region_realign, best_hap); F(phmm_region_realign, sw); F(phmm_region_realign, cigars);
    F(phmm_region_realign, cigar_capacity); F(phmm_region_realign, cigar_total);
    S(phmm_server_stats);
    F(phmm_server_stats, requests_submitted); F(phmm_server_stats, requests_done); F(phmm_server_stats, batches);
    F(phmm_server_stats, max_batch_regions); F(phmm_server_stats, queue_peak); F(phmm_server_stats, cells_done);
    F(phmm_server_stats, batch_ms); F(phmm_server_stats, device_ms); F(phmm_server_stats, max_batch_ms);
    F(phmm_server_stats, max_queue_ms); F(phmm_server_stats, arena_grows); F(phmm_server_stats, graph_captures);
    F(phmm_server_stats, max_setup_ms); F(phmm_server_stats, max_host_ms); F(phmm_server_stats, gather_ms);
    F(phmm_server_stats, plan_ms); F(phmm_server_stats, enqueue_ms); F(phmm_server_stats, wait_ms);
    F(phmm_server_stats, scatter_ms);
    S(phmm_sw_item);
    F(phmm_sw_item, hap_offset); F(phmm_sw_item, read_offset); F(phmm_sw_item, hap_len); F(phmm_sw_item, read_len);
    S(phmm_sw_result);
    F(phmm_sw_result, score); F(phmm_sw_result, alignment_offset); F(phmm_sw_result, max_i); F(phmm_sw_result, max_j);
    F(phmm_sw_result, cigar_count); F(phmm_sw_result, cigar_offset);
    return 0;
}
