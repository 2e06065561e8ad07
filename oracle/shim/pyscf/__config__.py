fci_csf_FCI_pspace_size = 200
