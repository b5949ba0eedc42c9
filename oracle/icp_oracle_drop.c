/* icp_oracle_drop.c -- CPU restatement of the drop path (filled in with the drop tracer).
 * TEST INFRASTRUCTURE ONLY. */
int icpo_drop_placeholder(void) { return 0; }
