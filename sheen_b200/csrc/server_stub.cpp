namespace sheen { void release_all_servers() {} }
